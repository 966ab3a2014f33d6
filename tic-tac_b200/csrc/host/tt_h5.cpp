// P123 files in the reference's HDF5 layout without libhdf5 (see tt_h5.h).
// The byte layouts below follow the published HDF5 file format
// specification (superblock version 0, version-1 object headers, symbol-table
// groups, datatype/dataspace/fill-value/layout/attribute messages).
#include "tt_h5.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>

namespace tt {

const char* const kPwFieldNames[kPwFields] = {"index", "L_12", "S_12", "J_12", "T_12",
                                              "l_3", "2*j_3", "2*T_total", "2*J_total", "PAR_total"};

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 8;       // a symbol-table node holds 2K = 16 links (the file has 10)
constexpr int kInternalK = 16;  // the library default for group B-trees
constexpr size_t kSnodSize = 8 + 2 * kLeafK * 40;
constexpr size_t kTreeSize = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;

// reference struct layouts (CPP/type_defs.h:126-137, 157-160): the tables'
// compound types carry these byte offsets, in the writer's field order
constexpr uint32_t kPwRecord = 40;
constexpr uint32_t kPwOffset[kPwFields] = {0, 4, 8, 12, 16, 20, 24, 36, 28, 32};
constexpr uint32_t kBoundsRecord = 16;

inline size_t round8(size_t n) { return (n + 7) & ~size_t(7); }

struct Bytes {
  std::vector<uint8_t> b;
  void u8(unsigned v) { b.push_back((uint8_t)v); }
  void u16(unsigned v) { u8(v & 0xff); u8((v >> 8) & 0xff); }
  void u32(uint32_t v) {
    for (int i = 0; i < 4; i++) u8((v >> (8 * i)) & 0xff);
  }
  void u64(uint64_t v) {
    for (int i = 0; i < 8; i++) u8((unsigned)((v >> (8 * i)) & 0xff));
  }
  void raw(const void* p, size_t n) {
    const uint8_t* q = (const uint8_t*)p;
    b.insert(b.end(), q, q + n);
  }
  void raw(const Bytes& o) { raw(o.b.data(), o.b.size()); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  // NUL-terminated name whose length (with the NUL) is padded to 8 bytes
  void name8(const std::string& s) {
    raw(s.data(), s.size());
    zeros(round8(s.size() + 1) - s.size());
  }
  size_t size() const { return b.size(); }
};

// ---- datatype messages (version 1 encodings) ----
Bytes dt_int(uint32_t bytes, bool is_signed) {
  Bytes d;
  d.u8(0x10 | 0);
  d.u8(is_signed ? 0x08 : 0x00);  // little endian, zero padding
  d.u8(0);
  d.u8(0);
  d.u32(bytes);
  d.u16(0);  // bit offset
  d.u16(8 * bytes);
  return d;
}
Bytes dt_f64() {
  Bytes d;
  d.u8(0x10 | 1);
  d.u8(0x20);  // little endian, implied leading mantissa bit
  d.u8(63);    // sign bit position
  d.u8(0);
  d.u32(8);
  d.u16(0);
  d.u16(64);
  d.u8(52);  // exponent location, size
  d.u8(11);
  d.u8(0);  // mantissa location, size
  d.u8(52);
  d.u32(1023);
  return d;
}
Bytes dt_str(uint32_t bytes) {
  Bytes d;
  d.u8(0x10 | 3);
  d.u8(0);  // NUL-terminated, ASCII
  d.u8(0);
  d.u8(0);
  d.u32(bytes);
  return d;
}
struct Member {
  std::string name;
  uint32_t offset;
  Bytes type;
};
Bytes dt_compound(uint32_t size, const std::vector<Member>& m) {
  Bytes d;
  d.u8(0x10 | 6);
  d.u8(m.size() & 0xff);
  d.u8((m.size() >> 8) & 0xff);
  d.u8(0);
  d.u32(size);
  for (const Member& x : m) {
    d.name8(x.name);
    d.u32(x.offset);
    d.u8(0);  // scalar member
    d.zeros(3);
    d.u32(0);  // permutation
    d.u32(0);
    d.zeros(16);  // dimension sizes
    d.raw(x.type);
  }
  return d;
}

// ---- dataspace, fill value, layout, attribute messages ----
Bytes ds_simple(uint64_t n) {
  Bytes d;
  d.u8(1);
  d.u8(1);  // rank
  d.u8(0);  // no maximum dimensions
  d.u8(0);
  d.u32(0);
  d.u64(n);
  return d;
}
Bytes ds_scalar() {
  Bytes d;
  d.u8(1);
  d.u8(0);
  d.u8(0);
  d.u8(0);
  d.u32(0);
  return d;
}
Bytes fill_msg() {
  Bytes d;
  d.u8(2);  // version
  d.u8(2);  // space allocated late
  d.u8(2);  // fill written if set
  d.u8(0);  // no fill value defined
  return d;
}
Bytes layout_contig(uint64_t addr, uint64_t size) {
  Bytes d;
  d.u8(3);
  d.u8(1);
  d.u64(addr);
  d.u64(size);
  return d;
}
Bytes attr_string(const std::string& name, const std::string& value) {
  const Bytes t = dt_str((uint32_t)value.size() + 1), s = ds_scalar();
  Bytes a;
  a.u8(1);
  a.u8(0);
  a.u16((unsigned)name.size() + 1);
  a.u16((unsigned)t.size());
  a.u16((unsigned)s.size());
  a.name8(name);
  a.raw(t);
  a.zeros(round8(t.size()) - t.size());
  a.raw(s);
  a.zeros(round8(s.size()) - s.size());
  a.raw(value.data(), value.size());
  a.u8(0);
  return a;
}

struct Msg {
  uint16_t type;
  Bytes data;
  uint8_t flags;
};
Bytes object_header(const std::vector<Msg>& msgs) {
  size_t body = 0;
  for (const Msg& m : msgs) body += 8 + round8(m.data.size());
  Bytes h;
  h.u8(1);  // version
  h.u8(0);
  h.u16((unsigned)msgs.size());
  h.u32(1);  // reference count
  h.u32((uint32_t)body);
  h.u32(0);  // alignment of the first message
  for (const Msg& m : msgs) {
    h.u16(m.type);
    h.u16((unsigned)round8(m.data.size()));
    h.u8(m.flags);
    h.zeros(3);
    h.raw(m.data);
    h.zeros(round8(m.data.size()) - m.data.size());
  }
  return h;
}

struct DatasetSpec {
  std::string name;
  Bytes type;
  Bytes space;
  uint64_t data_size = 0;
  const void* data = nullptr;  // data_size bytes
  std::vector<uint8_t> own;    // small payloads built here
  std::vector<std::pair<std::string, std::string>> attrs;
  Bytes header(uint64_t addr) const {
    std::vector<Msg> m;
    m.push_back({0x0001, space, 0});
    m.push_back({0x0003, type, 1});
    m.push_back({0x0005, fill_msg(), 1});
    m.push_back({0x0008, layout_contig(data_size ? addr : kUndef, data_size), 0});
    for (const auto& a : attrs) m.push_back({0x000C, attr_string(a.first, a.second), 0});
    return object_header(m);
  }
};

std::vector<DatasetSpec> p123_datasets(const P123H5& f, const int32_t* row, const int32_t* col, const double* val) {
  std::vector<DatasetSpec> d;
  auto scalar_int = [&](const char* name, int v) {
    DatasetSpec s;
    s.name = name;
    s.type = dt_int(4, true);
    s.space = ds_simple(1);
    s.own.resize(4);
    const int32_t x = v;
    std::memcpy(s.own.data(), &x, 4);
    s.data_size = 4;
    d.push_back(std::move(s));
  };
  scalar_int("Nalpha", f.Nalpha);
  scalar_int("Np_WP", f.Np_WP);
  scalar_int("Nq_WP", f.Nq_WP);
  {
    DatasetSpec s;
    s.name = "P123_sparse_dim";
    s.type = dt_int(8, false);
    s.space = ds_simple(1);
    s.own.resize(8);
    std::memcpy(s.own.data(), &f.nnz, 8);
    s.data_size = 8;
    d.push_back(std::move(s));
  }
  auto bounds = [&](const char* name, const char* title, const std::vector<double>& b) {
    DatasetSpec s;
    s.name = name;
    s.type = dt_compound(kBoundsRecord, {{"index", 0, dt_int(4, true)}, {"mesh point", 8, dt_f64()}});
    s.space = ds_simple(b.size());
    s.own.assign(b.size() * kBoundsRecord, 0);
    for (size_t i = 0; i < b.size(); i++) {
      const int32_t ix = (int32_t)i;
      std::memcpy(&s.own[i * kBoundsRecord], &ix, 4);
      std::memcpy(&s.own[i * kBoundsRecord + 8], &b[i], 8);
    }
    s.data_size = s.own.size();
    s.attrs = {{"CLASS", "TABLE"}, {"VERSION", "3.0"}, {"TITLE", title},
               {"FIELD_0_NAME", "index"}, {"FIELD_1_NAME", "mesh point"}};
    d.push_back(std::move(s));
  };
  bounds("p boundaries", "Info p boundaries", f.p_WP);
  bounds("q boundaries", "Info q boundaries", f.q_WP);
  {
    DatasetSpec s;
    s.name = "pw channels";
    std::vector<Member> m;
    for (int k = 0; k < kPwFields; k++) m.push_back({kPwFieldNames[k], kPwOffset[k], dt_int(4, true)});
    s.type = dt_compound(kPwRecord, m);
    s.space = ds_simple((uint64_t)f.Nalpha);
    s.own.assign((size_t)f.Nalpha * kPwRecord, 0);
    for (int a = 0; a < f.Nalpha; a++)
      for (int k = 0; k < kPwFields; k++) std::memcpy(&s.own[a * kPwRecord + kPwOffset[k]], &f.pw[a * kPwFields + k], 4);
    s.data_size = s.own.size();
    s.attrs = {{"CLASS", "TABLE"}, {"VERSION", "3.0"}, {"TITLE", "Partial wave info"}};
    for (int k = 0; k < kPwFields; k++) s.attrs.push_back({"FIELD_" + std::to_string(k) + "_NAME", kPwFieldNames[k]});
    d.push_back(std::move(s));
  }
  auto big = [&](const char* name, Bytes type, const void* p, size_t elem) {
    DatasetSpec s;
    s.name = name;
    s.type = std::move(type);
    s.space = ds_simple(f.nnz);
    s.data = p;
    s.data_size = f.nnz * elem;
    d.push_back(std::move(s));
  };
  big("row indices", dt_int(4, true), row, 4);
  big("column indices", dt_int(4, true), col, 4);
  big("values", dt_f64(), val, 8);
  return d;
}

}  // namespace

static bool write_p123(const std::string& path, const P123H5& f, const int32_t* row, const int32_t* col,
                       const double* val, std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return false;
  };
  if (f.Nalpha <= 0 || f.Np_WP <= 0 || f.Nq_WP <= 0) return fail("P123 file: empty state space");
  if ((int)f.p_WP.size() != f.Np_WP + 1 || (int)f.q_WP.size() != f.Nq_WP + 1)
    return fail("P123 file: boundary arrays must hold N+1 values");
  if ((int64_t)f.pw.size() != (int64_t)f.Nalpha * kPwFields) return fail("P123 file: pw table size");
  if (!row) row = f.row.data();
  if (!col) col = f.col.data();
  if (!val) val = f.val.data();
  if (f.nnz && (!row || !col || !val)) return fail("P123 file: missing sparse arrays");
  std::vector<DatasetSpec> ds = p123_datasets(f, row, col, val);
  std::sort(ds.begin(), ds.end(), [](const DatasetSpec& a, const DatasetSpec& b) { return a.name < b.name; });

  // local heap: "" at offset 0, then the link names
  Bytes heap_data;
  heap_data.zeros(8);
  std::vector<uint64_t> name_off;
  for (const auto& d : ds) {
    name_off.push_back(heap_data.size());
    heap_data.name8(d.name);
  }
  // addresses, in file order
  const uint64_t a_root = 96;
  const Bytes root_probe = object_header({{0x0011, Bytes{std::vector<uint8_t>(16, 0)}, 0}});
  const uint64_t a_heap = a_root + root_probe.size();
  const uint64_t a_heap_data = a_heap + 32;
  const uint64_t a_tree = a_heap_data + heap_data.size();
  const uint64_t a_snod = a_tree + kTreeSize;
  uint64_t a = a_snod + kSnodSize;
  std::vector<uint64_t> a_oh(ds.size()), a_data(ds.size());
  for (size_t i = 0; i < ds.size(); i++) {
    a_oh[i] = a;
    a += ds[i].header(0).size();
  }
  for (size_t i = 0; i < ds.size(); i++) {
    a_data[i] = a;
    a += round8(ds[i].data_size);
  }
  const uint64_t eof = a;

  Bytes m;  // all metadata, addresses [0, a_data[0])
  // superblock version 0
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  m.raw(sig, 8);
  m.u8(0);  // superblock
  m.u8(0);  // free space
  m.u8(0);  // root symbol table entry
  m.u8(0);
  m.u8(0);  // shared header messages
  m.u8(8);  // size of offsets
  m.u8(8);  // size of lengths
  m.u8(0);
  m.u16(kLeafK);
  m.u16(kInternalK);
  m.u32(0);  // consistency flags
  m.u64(0);  // base address
  m.u64(kUndef);
  m.u64(eof);
  m.u64(kUndef);
  // root group symbol table entry: cached B-tree and heap addresses
  m.u64(0);
  m.u64(a_root);
  m.u32(1);
  m.u32(0);
  m.u64(a_tree);
  m.u64(a_heap);
  // root object header: the symbol table message
  {
    Bytes st;
    st.u64(a_tree);
    st.u64(a_heap);
    m.raw(object_header({{0x0011, st, 0}}));
  }
  // local heap
  m.raw("HEAP", 4);
  m.u8(0);
  m.zeros(3);
  m.u64(heap_data.size());
  m.u64(1);  // no free block
  m.u64(a_heap_data);
  m.raw(heap_data);
  // group B-tree: one leaf pointing at one symbol-table node
  {
    Bytes t;
    t.raw("TREE", 4);
    t.u8(0);  // group node
    t.u8(0);  // leaf level
    t.u16(1);
    t.u64(kUndef);
    t.u64(kUndef);
    t.u64(0);  // key 0: the empty name
    t.u64(a_snod);
    t.u64(name_off.back());  // key 1: the largest name in the node
    t.zeros(kTreeSize - t.size());
    m.raw(t);
  }
  {
    Bytes s;
    s.raw("SNOD", 4);
    s.u8(1);
    s.u8(0);
    s.u16((unsigned)ds.size());
    for (size_t i = 0; i < ds.size(); i++) {
      s.u64(name_off[i]);
      s.u64(a_oh[i]);
      s.u32(0);
      s.u32(0);
      s.zeros(16);
    }
    s.zeros(kSnodSize - s.size());
    m.raw(s);
  }
  for (size_t i = 0; i < ds.size(); i++) m.raw(ds[i].header(a_data[i]));
  if (m.size() != a_data[0]) return fail("P123 file: internal layout error");

  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return fail("cannot create " + path);
  bool ok = std::fwrite(m.b.data(), 1, m.size(), fp) == m.size();
  const uint8_t zero[8] = {0};
  for (size_t i = 0; ok && i < ds.size(); i++) {
    const void* p = ds[i].data ? ds[i].data : ds[i].own.data();
    if (ds[i].data_size) ok = std::fwrite(p, 1, ds[i].data_size, fp) == ds[i].data_size;
    const size_t pad = round8(ds[i].data_size) - ds[i].data_size;
    if (ok && pad) ok = std::fwrite(zero, 1, pad, fp) == pad;
  }
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) return fail("write to " + path + " failed");
  return true;
}

// ======================================================================
// reader
// ======================================================================
namespace {

struct Cur {
  const uint8_t* p;
  const uint8_t* e;
  bool ok = true;
  Cur(const uint8_t* a, size_t n) : p(a), e(a + n) {}
  bool need(size_t n) {
    if ((size_t)(e - p) < n) ok = false;
    return ok;
  }
  uint64_t un(int n) {
    if (!need(n)) return 0;
    uint64_t v = 0;
    for (int i = 0; i < n; i++) v |= (uint64_t)p[i] << (8 * i);
    p += n;
    return v;
  }
  unsigned u8() { return (unsigned)un(1); }
  unsigned u16() { return (unsigned)un(2); }
  uint32_t u32() { return (uint32_t)un(4); }
  uint64_t u64() { return un(8); }
  void skip(size_t n) {
    if (need(n)) p += n;
  }
  std::string cstr() {
    const uint8_t* q = p;
    while (q < e && *q) q++;
    if (q == e) {
      ok = false;
      return {};
    }
    std::string s((const char*)p, q - p);
    p = q + 1;
    return s;
  }
};

struct DType {
  int cls = -1;
  uint32_t size = 0;
  bool is_signed = false;
  bool big_endian = false;
  // compound members (std::vector allows the incomplete element type)
  std::vector<std::string> mname;
  std::vector<uint32_t> moff;
  std::vector<DType> mtype;
};

bool parse_dtype(Cur& c, DType& t) {
  const unsigned cv = c.u8();
  const unsigned version = cv >> 4;
  t.cls = cv & 0x0f;
  const unsigned b0 = c.u8(), b1 = c.u8(), b2 = c.u8();
  t.size = c.u32();
  if (!c.ok) return false;
  switch (t.cls) {
    case 0:  // fixed point
      t.big_endian = b0 & 1;
      t.is_signed = (b0 >> 3) & 1;
      c.skip(4);
      break;
    case 1:  // floating point
      t.big_endian = b0 & 1;
      c.skip(12);
      break;
    case 3:  // string
      break;
    case 6: {  // compound
      const unsigned nm = b0 | (b1 << 8);
      (void)b2;
      for (unsigned i = 0; i < nm && c.ok; i++) {
        const uint8_t* start = c.p;
        t.mname.push_back(c.cstr());
        if (version < 3) {
          const size_t used = c.p - start;
          c.skip(round8(used) - used);
          t.moff.push_back(c.u32());
          if (version == 1) c.skip(1 + 3 + 4 + 4 + 16);
        } else {
          int nb = 1;
          while (nb < 4 && (uint64_t(1) << (8 * nb)) <= t.size) nb++;
          t.moff.push_back((uint32_t)c.un(nb));
        }
        t.mtype.emplace_back();
        if (!parse_dtype(c, t.mtype.back())) return false;
      }
      break;
    }
    default:
      return false;
  }
  return c.ok;
}

struct Layout {
  int cls = -1;
  uint64_t addr = kUndef, size = 0;
  std::vector<uint8_t> compact;
  std::vector<uint32_t> chunk;  // chunked: dims incl. the element size
};

struct Dataset {
  std::vector<uint64_t> dims;
  DType type;
  Layout layout;
  bool filtered = false;
};

class Reader {
 public:
  std::string err;
  ~Reader() {
    if (fp_) std::fclose(fp_);
  }
  bool open(const std::string& path) {
    fp_ = std::fopen(path.c_str(), "rb");
    if (!fp_) return fail("cannot open " + path);
    std::fseek(fp_, 0, SEEK_END);
    fsize_ = (uint64_t)std::ftell(fp_);
    uint8_t sb[104];
    if (!rd(0, sb, std::min<uint64_t>(sizeof sb, fsize_))) return false;
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    if (fsize_ < 96 || std::memcmp(sb, sig, 8) != 0) return fail(path + " is not an HDF5 file");
    const unsigned v = sb[8];
    if (v > 1) return fail("HDF5 superblock version " + std::to_string(v) + " is not supported");
    if (sb[13] != 8 || sb[14] != 8) return fail("HDF5 file with offsets/lengths other than 8 bytes");
    Cur c(sb + 24 + (v == 1 ? 4 : 0), 48);
    c.u64();  // base address
    c.u64();
    c.u64();  // end of file
    c.u64();
    c.u64();  // link name offset
    root_ = c.u64();
    return c.ok || fail("truncated superblock");
  }
  // root group links: name -> object header address
  bool root_links(std::map<std::string, uint64_t>& out) {
    std::vector<std::pair<uint16_t, std::vector<uint8_t>>> msgs;
    if (!header(root_, msgs)) return false;
    for (auto& m : msgs)
      if (m.first == 0x0011) {
        Cur c(m.second.data(), m.second.size());
        const uint64_t tree = c.u64(), heap = c.u64();
        std::vector<uint8_t> names;
        if (!local_heap(heap, names)) return false;
        return group_tree(tree, names, out, 0);
      }
    return fail("root group has no symbol table (newer group format not supported)");
  }
  bool dataset(uint64_t oh, Dataset& d) {
    std::vector<std::pair<uint16_t, std::vector<uint8_t>>> msgs;
    if (!header(oh, msgs)) return false;
    bool have_space = false, have_type = false;
    for (auto& m : msgs) {
      Cur c(m.second.data(), m.second.size());
      if (m.first == 0x0001) {
        const unsigned ver = c.u8(), rank = c.u8(), flags = c.u8();
        if (ver == 1)
          c.skip(5);
        else
          c.skip(1);
        d.dims.clear();
        for (unsigned i = 0; i < rank; i++) d.dims.push_back(c.u64());
        (void)flags;
        have_space = c.ok;
      } else if (m.first == 0x0003) {
        have_type = parse_dtype(c, d.type);
      } else if (m.first == 0x0008) {
        const unsigned ver = c.u8();
        if (ver != 3) return fail("data layout message version " + std::to_string(ver) + " is not supported");
        d.layout.cls = (int)c.u8();
        if (d.layout.cls == 0) {
          const unsigned n = c.u16();
          if (c.need(n)) d.layout.compact.assign(c.p, c.p + n);
        } else if (d.layout.cls == 1) {
          d.layout.addr = c.u64();
          d.layout.size = c.u64();
        } else if (d.layout.cls == 2) {
          const unsigned nd = c.u8();
          d.layout.addr = c.u64();
          for (unsigned i = 0; i < nd; i++) d.layout.chunk.push_back(c.u32());
        }
        if (!c.ok) return fail("truncated layout message");
      } else if (m.first == 0x000B) {
        d.filtered = true;
      }
    }
    if (!have_space || !have_type || d.layout.cls < 0) return fail("incomplete dataset object header");
    if (d.filtered) return fail("filtered (compressed) datasets are not supported");
    return true;
  }
  // the dataset's raw elements (row-major), type size bytes each
  bool data(const Dataset& d, std::vector<uint8_t>& out) {
    // unfiltered data never exceeds the file: bound the extent before allocating
    uint64_t n = 1;
    for (uint64_t x : d.dims) {
      if (x != 0 && n > fsize_ / x) return fail("dataset extent larger than the file");
      n *= x;
    }
    if (d.type.size == 0 || (n != 0 && d.type.size > fsize_ / n)) return fail("dataset larger than the file");
    const uint64_t bytes = n * d.type.size;
    out.assign(bytes, 0);
    if (d.layout.cls == 0) {
      if (d.layout.compact.size() < bytes) return fail("short compact dataset");
      std::memcpy(out.data(), d.layout.compact.data(), bytes);
      return true;
    }
    if (d.layout.cls == 1) {
      if (d.layout.addr == kUndef) return true;  // never written: fill (zero)
      if (d.layout.size < bytes) return fail("short contiguous dataset");
      return rd(d.layout.addr, out.data(), bytes);
    }
    if (d.layout.cls == 2) {
      if (d.dims.size() != 1 || d.layout.chunk.size() != 2) return fail("only rank-1 chunked datasets are supported");
      if (d.layout.addr == kUndef) return true;
      return chunk_tree(d.layout.addr, d, out, 0);
    }
    return fail("unknown storage layout");
  }

 private:
  FILE* fp_ = nullptr;
  uint64_t fsize_ = 0, root_ = kUndef;
  bool fail(const std::string& m) {
    err = m;
    return false;
  }
  bool rd(uint64_t addr, void* p, uint64_t n) {
    if (addr > fsize_ || n > fsize_ - addr) return fail("HDF5 structure points beyond the end of the file");
    if (std::fseek(fp_, (long)addr, SEEK_SET) != 0 || std::fread(p, 1, n, fp_) != n) return fail("read failed");
    return true;
  }
  bool header(uint64_t addr, std::vector<std::pair<uint16_t, std::vector<uint8_t>>>& msgs) {
    uint8_t pre[16];
    if (!rd(addr, pre, 16)) return false;
    if (pre[0] != 1) return fail("object header version " + std::to_string(pre[0]) + " is not supported");
    Cur c(pre, 16);
    c.skip(2);
    const unsigned nmsg = c.u16();
    c.u32();
    const uint32_t size = c.u32();
    std::vector<std::pair<uint64_t, uint64_t>> chunks{{addr + 16, size}};
    unsigned seen = 0;
    for (size_t k = 0; k < chunks.size() && k < 64; k++) {
      if (chunks[k].second > fsize_) return fail("object header block larger than the file");
      std::vector<uint8_t> b(chunks[k].second);
      if (!rd(chunks[k].first, b.data(), b.size())) return false;
      Cur m(b.data(), b.size());
      while (m.ok && (size_t)(m.e - m.p) >= 8 && seen < nmsg) {
        const unsigned type = m.u16(), len = m.u16();
        m.skip(4);
        if (!m.need(len)) return fail("truncated object header message");
        std::vector<uint8_t> body(m.p, m.p + len);
        m.p += len;
        seen++;
        if (type == 0x0010) {
          Cur q(body.data(), body.size());
          const uint64_t off = q.u64(), n = q.u64();
          chunks.push_back({off, n});
        } else if (type != 0) {
          msgs.push_back({(uint16_t)type, std::move(body)});
        }
      }
    }
    return true;
  }
  bool local_heap(uint64_t addr, std::vector<uint8_t>& data) {
    uint8_t h[32];
    if (!rd(addr, h, 32)) return false;
    if (std::memcmp(h, "HEAP", 4) != 0) return fail("bad local heap signature");
    Cur c(h + 8, 24);
    const uint64_t size = c.u64();
    c.u64();
    const uint64_t a = c.u64();
    if (size > fsize_) return fail("local heap larger than the file");
    data.resize(size);
    return rd(a, data.data(), size);
  }
  bool group_tree(uint64_t addr, const std::vector<uint8_t>& names, std::map<std::string, uint64_t>& out, int depth) {
    if (depth > 16) return fail("group B-tree too deep");
    uint8_t h[24];
    if (!rd(addr, h, 24)) return false;
    if (std::memcmp(h, "TREE", 4) != 0 || h[4] != 0) return fail("bad group B-tree node");
    const unsigned level = h[5], entries = h[6] | (h[7] << 8);
    std::vector<uint8_t> b((size_t)entries * 16 + 8);
    if (!rd(addr + 24, b.data(), b.size())) return false;
    Cur c(b.data(), b.size());
    for (unsigned i = 0; i < entries; i++) {
      c.u64();  // key
      const uint64_t child = c.u64();
      if (level > 0) {
        if (!group_tree(child, names, out, depth + 1)) return false;
      } else if (!symbol_node(child, names, out)) {
        return false;
      }
    }
    return true;
  }
  bool symbol_node(uint64_t addr, const std::vector<uint8_t>& names, std::map<std::string, uint64_t>& out) {
    uint8_t h[8];
    if (!rd(addr, h, 8)) return false;
    if (std::memcmp(h, "SNOD", 4) != 0) return fail("bad symbol table node");
    const unsigned n = h[6] | (h[7] << 8);
    std::vector<uint8_t> b((size_t)n * 40);
    if (!rd(addr + 8, b.data(), b.size())) return false;
    Cur c(b.data(), b.size());
    for (unsigned i = 0; i < n; i++) {
      const uint64_t off = c.u64(), oh = c.u64();
      c.skip(24);
      if (off >= names.size()) return fail("link name outside the local heap");
      const char* s = (const char*)names.data() + off;
      out[std::string(s, strnlen(s, names.size() - off))] = oh;
    }
    return true;
  }
  bool chunk_tree(uint64_t addr, const Dataset& d, std::vector<uint8_t>& out, int depth) {
    if (depth > 16) return fail("chunk B-tree too deep");
    uint8_t h[24];
    if (!rd(addr, h, 24)) return false;
    if (std::memcmp(h, "TREE", 4) != 0 || h[4] != 1) return fail("bad chunk B-tree node");
    const unsigned level = h[5], entries = h[6] | (h[7] << 8);
    const size_t key = 8 + 8 * d.layout.chunk.size();
    std::vector<uint8_t> b((size_t)entries * (key + 8) + key);
    if (!rd(addr + 24, b.data(), b.size())) return false;
    Cur c(b.data(), b.size());
    const uint64_t esz = d.type.size, cdim = d.layout.chunk[0];
    for (unsigned i = 0; i < entries; i++) {
      const uint32_t nbytes = c.u32(), mask = c.u32();
      const uint64_t off = c.u64();
      c.u64();  // element-size dimension
      const uint64_t child = c.u64();
      if (level > 0) {
        if (!chunk_tree(child, d, out, depth + 1)) return false;
        continue;
      }
      if (mask != 0) return fail("filtered chunk");
      if (off >= d.dims[0]) continue;
      const uint64_t count = std::min<uint64_t>(cdim, d.dims[0] - off);
      if ((uint64_t)nbytes < count * esz) return fail("short chunk");
      if (!rd(child, out.data() + off * esz, count * esz)) return false;
    }
    return true;
  }
};

bool le_scalar_ok(const DType& t, int cls, uint32_t size) { return t.cls == cls && t.size == size && !t.big_endian; }

// elements of a fixed-point dataset (or compound member) as int64
bool to_i64(const DType& t, const uint8_t* p, int64_t& v) {
  if (t.cls != 0 || t.big_endian || (t.size != 4 && t.size != 8)) return false;
  if (t.size == 4) {
    uint32_t u;
    std::memcpy(&u, p, 4);
    v = t.is_signed ? (int64_t)(int32_t)u : (int64_t)u;
  } else {
    uint64_t u;
    std::memcpy(&u, p, 8);
    v = (int64_t)u;
  }
  return true;
}

}  // namespace

static bool read_p123(const std::string& path, P123H5& f, std::string* err) {
  Reader r;
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return false;
  };
  if (!r.open(path)) return fail(r.err);
  std::map<std::string, uint64_t> links;
  if (!r.root_links(links)) return fail(r.err);
  auto get = [&](const char* name, Dataset& d, std::vector<uint8_t>* raw) -> bool {
    auto it = links.find(name);
    if (it == links.end()) return fail(path + ": no dataset \"" + name + "\"");
    if (!r.dataset(it->second, d)) return fail(path + ": \"" + name + "\": " + r.err);
    if (d.dims.size() != 1) return fail(path + ": \"" + name + "\" is not one-dimensional");
    if (raw && !r.data(d, *raw)) return fail(path + ": \"" + name + "\": " + r.err);
    return true;
  };
  auto scalar = [&](const char* name, int64_t& v) -> bool {
    Dataset d;
    std::vector<uint8_t> raw;
    if (!get(name, d, &raw)) return false;
    if (d.dims[0] != 1 || !to_i64(d.type, raw.data(), v)) return fail(path + ": \"" + name + "\" is not an integer[1]");
    return true;
  };
  int64_t na, np, nq, nnz;
  if (!scalar("Nalpha", na) || !scalar("Np_WP", np) || !scalar("Nq_WP", nq) || !scalar("P123_sparse_dim", nnz))
    return false;
  if (na <= 0 || np <= 0 || nq <= 0 || nnz < 0 || na > (1 << 20) || np > (1 << 20) || nq > (1 << 20))
    return fail(path + ": implausible dimensions");
  f.Nalpha = (int)na;
  f.Np_WP = (int)np;
  f.Nq_WP = (int)nq;
  f.nnz = (uint64_t)nnz;
  // index of the compound member called name, or -1
  auto member = [](const DType& t, const char* name) -> int {
    for (size_t i = 0; i < t.mname.size(); i++)
      if (t.mname[i] == name) return (int)i;
    return -1;
  };
  auto bounds = [&](const char* name, int N, std::vector<double>& b) -> bool {
    Dataset d;
    std::vector<uint8_t> raw;
    if (!get(name, d, &raw)) return false;
    const int mi = d.type.cls == 6 ? member(d.type, "mesh point") : -1;
    if (mi < 0 || !le_scalar_ok(d.type.mtype[mi], 1, 8) || d.type.moff[mi] + 8 > d.type.size)
      return fail(path + ": \"" + name + "\" has no float64 field \"mesh point\"");
    if (d.dims[0] != (uint64_t)N + 1) return fail(path + ": \"" + name + "\" does not hold N+1 boundaries");
    b.resize(N + 1);
    for (int i = 0; i <= N; i++) std::memcpy(&b[i], raw.data() + (size_t)i * d.type.size + d.type.moff[mi], 8);
    return true;
  };
  if (!bounds("p boundaries", f.Np_WP, f.p_WP) || !bounds("q boundaries", f.Nq_WP, f.q_WP)) return false;
  {
    Dataset d;
    std::vector<uint8_t> raw;
    if (!get("pw channels", d, &raw)) return false;
    if (d.type.cls != 6 || d.dims[0] != (uint64_t)f.Nalpha)
      return fail(path + ": \"pw channels\" is not a table of Nalpha records");
    f.pw.assign((size_t)f.Nalpha * kPwFields, 0);
    for (int k = 0; k < kPwFields; k++) {
      const int mi = member(d.type, kPwFieldNames[k]);
      if (mi < 0 || d.type.mtype[mi].cls != 0 || d.type.moff[mi] + d.type.mtype[mi].size > d.type.size)
        return fail(path + ": \"pw channels\" has no integer field \"" + kPwFieldNames[k] + "\"");
      for (int a = 0; a < f.Nalpha; a++) {
        int64_t v;
        if (!to_i64(d.type.mtype[mi], raw.data() + (size_t)a * d.type.size + d.type.moff[mi], v))
          return fail(path + ": \"pw channels\" field type");
        f.pw[(size_t)a * kPwFields + k] = (int32_t)v;
      }
    }
  }
  auto sparse = [&](const char* name, int cls, void* dst) -> bool {
    Dataset d;
    if (!get(name, d, nullptr)) return false;
    if (d.dims[0] != f.nnz) return fail(path + ": \"" + name + "\" length differs from P123_sparse_dim");
    if (!le_scalar_ok(d.type, cls, cls == 1 ? 8 : 4) || (cls == 0 && !d.type.is_signed))
      return fail(path + ": \"" + name + "\" has an unexpected datatype");
    std::vector<uint8_t> raw;
    if (!r.data(d, raw)) return fail(path + ": \"" + name + "\": " + r.err);
    if (!raw.empty()) std::memcpy(dst, raw.data(), raw.size());
    return true;
  };
  f.row.resize(f.nnz);
  f.col.resize(f.nnz);
  f.val.resize(f.nnz);
  if (!sparse("row indices", 0, f.row.data()) || !sparse("column indices", 0, f.col.data()) ||
      !sparse("values", 1, f.val.data()))
    return false;
  return true;
}

// host allocation failures become errors, never exceptions through the C ABI
bool h5_write_p123(const std::string& path, const P123H5& f, const int32_t* row, const int32_t* col,
                   const double* val, std::string* err) {
  try {
    return write_p123(path, f, row, col, val, err);
  } catch (const std::exception& e) {
    if (err) *err = std::string("P123 file: ") + e.what();
    return false;
  }
}

bool h5_read_p123(const std::string& path, P123H5& f, std::string* err) {
  try {
    return read_p123(path, f, err);
  } catch (const std::exception& e) {
    if (err) *err = path + ": " + e.what();
    return false;
  }
}

std::string p123_h5_filename(const std::string& folder, int two_J_3N, int P_3N, int Np_WP, int Nq_WP, int J_2N_max) {
  return folder + "/" + "P123_sparse_JP_" + std::to_string(two_J_3N) + "_" + std::to_string(P_3N) + "_Np_" +
         std::to_string(Np_WP) + "_Nq_" + std::to_string(Nq_WP) + "_J2max_" + std::to_string(J_2N_max) + ".h5";
}

}  // namespace tt
