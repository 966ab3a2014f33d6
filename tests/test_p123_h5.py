"""P123 files in the reference's HDF5 layout (tt_store_P123_h5 / tt_read_P123_h5).

No HDF5 library exists in this environment, so the library's files are
checked with an independent reader written from the file format
specification (tests/h5_spec.py), against the object list, datatypes, table
layouts and attributes of the reference's writer
(CPP/disk_io_routines.cpp:1078-1164, 1286-1545, 1625-1672), and the library's
reader is checked on files laid out the way the HDF5 library stores
H5TBmake_table tables (chunked, unlimited)."""
import numpy as np
import pytest

import h5_spec
import tictac_b200 as tt
from conftest import load_case

PW_FIELDS = ["index", "L_12", "S_12", "J_12", "T_12", "l_3", "2*j_3", "2*T_total", "2*J_total", "PAR_total"]
# byte offsets of those fields in the reference's pw_table struct (CPP/type_defs.h:126-137)
PW_OFFSETS = [0, 4, 8, 12, 16, 20, 24, 36, 28, 32]


def channel(name, c):
    g, m = load_case(name)
    pwt = g[f"pw_c{c}"]
    return dict(pwt=pwt, pw=tt.PW(pwt, J_2N_max=int(m["opts"].get("J_2N_max", 1))), p=g["p_WP"], q=g["q_WP"],
                row=g[f"p123_row_c{c}"], col=g[f"p123_col_c{c}"], val=g[f"p123_val_c{c}"])


def expected_pw_records(pwt):
    # pw_table rows as write_PW_statespace_to_h5 fills them (L S J T l 2j 2J 2T P columns in pwt)
    out = []
    for a, r in enumerate(np.asarray(pwt).reshape(-1, 9)):
        L, S, J, T, l, j2, J2, T2, P = (int(x) for x in r)
        out.append([a, L, S, J, T, l, j2, T2, int(pwt[0][6]), int(pwt[0][8])])
    return np.array(out, dtype=np.int32)


@pytest.mark.parametrize("case,c", [("lo_j1_J3_n8", 0), ("lo_j1_J3_n8", 3), ("mt_swave_n16", 0)])
def test_written_file_matches_reference_layout(tmp_path, case, c):
    ch = channel(case, c)
    path = tmp_path / "P123.h5"
    tt.store_P123_h5(path, ch["row"], ch["col"], ch["val"], ch["pw"], ch["p"], ch["q"])
    f = h5_spec.File(path)
    assert f.superblock_version == 0 and f.eof == path.stat().st_size
    assert sorted(f.datasets) == sorted(["Nalpha", "Np_WP", "Nq_WP", "P123_sparse_dim", "p boundaries",
                                         "q boundaries", "pw channels", "row indices", "column indices", "values"])
    d = f.datasets
    Nalpha = len(np.asarray(ch["pwt"]).reshape(-1, 9))
    for name, v in (("Nalpha", Nalpha), ("Np_WP", len(ch["p"]) - 1), ("Nq_WP", len(ch["q"]) - 1)):
        t = d[name]["type"]
        assert t["class"] == "int" and t["size"] == 4 and t["signed"] and d[name]["dims"] == [1]
        assert int(d[name]["data"][0]) == v
    t = d["P123_sparse_dim"]["type"]
    assert t["class"] == "int" and t["size"] == 8 and not t["signed"]
    assert int(d["P123_sparse_dim"]["data"][0]) == len(ch["val"])
    for name, b, title in (("p boundaries", ch["p"], "Info p boundaries"), ("q boundaries", ch["q"], "Info q boundaries")):
        t = d[name]["type"]
        assert t["class"] == "compound" and t["size"] == 16
        assert t["names"] == ["index", "mesh point"] and t["offsets"] == [0, 8]
        assert np.array_equal(d[name]["data"]["index"], np.arange(len(b)))
        assert np.array_equal(d[name]["data"]["mesh point"], b)  # bit-equal, the reader compares with !=
        assert d[name]["attrs"] == {"CLASS": "TABLE", "VERSION": "3.0", "TITLE": title,
                                   "FIELD_0_NAME": "index", "FIELD_1_NAME": "mesh point"}
    t = d["pw channels"]["type"]
    assert t["class"] == "compound" and t["size"] == 40
    assert t["names"] == PW_FIELDS and t["offsets"] == PW_OFFSETS
    recs = np.stack([d["pw channels"]["data"][k] for k in PW_FIELDS], axis=1)
    assert np.array_equal(recs, expected_pw_records(ch["pwt"]))
    attrs = d["pw channels"]["attrs"]
    assert attrs["CLASS"] == "TABLE" and attrs["TITLE"] == "Partial wave info"
    assert [attrs[f"FIELD_{k}_NAME"] for k in range(10)] == PW_FIELDS
    for name, ref, kind, size in (("row indices", ch["row"], "int", 4), ("column indices", ch["col"], "int", 4),
                                  ("values", ch["val"], "float", 8)):
        t = d[name]["type"]
        assert t["class"] == kind and t["size"] == size and t["np"].byteorder in "<="
        assert d[name]["layout"]["class"] == "contiguous"
        assert np.array_equal(d[name]["data"], ref)


def test_round_trip_and_reference_checks(tmp_path):
    ch = channel("lo_j1_J3_n8", 1)
    path = tmp_path / "P123.h5"
    tt.store_P123_h5(path, ch["row"], ch["col"], ch["val"], ch["pw"], ch["p"], ch["q"])
    r, c, v = tt.read_P123_h5(path, ch["pw"], ch["p"], ch["q"])
    assert np.array_equal(r, ch["row"]) and np.array_equal(c, ch["col"]) and np.array_equal(v, ch["val"])
    # the reference's integrity checks (CPP/disk_io_routines.cpp:1209-1270)
    p2 = np.array(ch["p"], dtype=np.float64)
    p2[3] = np.nextafter(p2[3], np.inf)
    with pytest.raises(tt.TicTacError, match="p-momentum boundaries mismatch"):
        tt.read_P123_h5(path, ch["pw"], p2, ch["q"])
    q2 = np.array(ch["q"], dtype=np.float64)
    q2[-1] *= 1 + 1e-15
    with pytest.raises(tt.TicTacError, match="q-momentum boundaries mismatch"):
        tt.read_P123_h5(path, ch["pw"], ch["p"], q2)
    with pytest.raises(tt.TicTacError, match="state-space dimensions"):
        tt.read_P123_h5(path, ch["pw"], ch["p"][:-1], ch["q"])
    pwt = np.array(ch["pwt"]).reshape(-1, 9).copy()
    pwt[-1, 4] += 2  # l_3 of the last state
    with pytest.raises(tt.TicTacError, match="PW state-space mismatch"):
        tt.read_P123_h5(path, tt.PW(pwt), ch["p"], ch["q"])
    with pytest.raises(tt.TicTacError):
        tt.read_P123_h5(tmp_path / "missing.h5", ch["pw"], ch["p"], ch["q"])


def test_corrupt_files_are_errors(tmp_path):
    ch = channel("lo_j1_J3_n8", 0)
    good = tmp_path / "good.h5"
    tt.store_P123_h5(good, ch["row"], ch["col"], ch["val"], ch["pw"], ch["p"], ch["q"])
    raw = good.read_bytes()
    rng = np.random.default_rng(5)
    cases = {"truncated": raw[:len(raw) // 2], "header only": raw[:96], "not hdf5": b"x" * 200}
    for i in range(8):  # random byte damage in the metadata (the first 2 KiB)
        b = bytearray(raw)
        for pos in rng.integers(8, 2048, size=4):
            b[pos] ^= 0xFF
        cases[f"damaged {i}"] = bytes(b)
    for name, data in cases.items():
        path = tmp_path / f"{name}.h5"
        path.write_bytes(data)
        try:
            r, c, v = tt.read_P123_h5(path, ch["pw"], ch["p"], ch["q"])
        except tt.TicTacError:
            continue  # a clean error
        # damage that misses every checked structure must still give the stored matrix
        assert len(r) == len(c) == len(v)


def test_empty_matrix(tmp_path):
    ch = channel("mt_swave_n16", 0)
    path = tmp_path / "empty.h5"
    e = np.zeros(0)
    tt.store_P123_h5(path, e.astype(np.int32), e.astype(np.int32), e, ch["pw"], ch["p"], ch["q"])
    f = h5_spec.File(path)
    assert f.datasets["values"]["dims"] == [0] and len(f.datasets["values"]["data"]) == 0
    r, c, v = tt.read_P123_h5(path, ch["pw"], ch["p"], ch["q"])
    assert len(r) == len(c) == len(v) == 0


def _library_style_file(path, ch, leaf_k, split=False):
    """The same objects with the tables chunked (10 records per chunk) and of
    unlimited maximum size, as H5TBmake_table stores them, the links spread
    over several symbol-table nodes, and (split) the table attributes in
    object-header continuation blocks."""
    pwt = np.asarray(ch["pwt"]).reshape(-1, 9)
    recs = expected_pw_records(ch["pwt"])
    pw_bytes = bytearray(40 * len(recs))
    for a, rec in enumerate(recs):
        for k, off in enumerate(PW_OFFSETS):
            pw_bytes[40 * a + off:40 * a + off + 4] = int(rec[k]).to_bytes(4, "little", signed=True)

    def bounds(b):
        out = bytearray(16 * len(b))
        for i, x in enumerate(b):
            out[16 * i:16 * i + 4] = i.to_bytes(4, "little")
            out[16 * i + 8:16 * i + 16] = np.float64(x).tobytes()
        return bytes(out)

    bt = h5_spec.dt_compound(16, [("index", 0, h5_spec.dt_int()), ("mesh point", 8, h5_spec.dt_f64())])
    pt = h5_spec.dt_compound(40, [(n, o, h5_spec.dt_int()) for n, o in zip(PW_FIELDS, PW_OFFSETS)])
    n = len(ch["val"])
    ds = [
        dict(name="Nalpha", type=h5_spec.dt_int(), n=1, data=np.int32(len(pwt)).tobytes()),
        dict(name="Np_WP", type=h5_spec.dt_int(), n=1, data=np.int32(len(ch["p"]) - 1).tobytes()),
        dict(name="Nq_WP", type=h5_spec.dt_int(), n=1, data=np.int32(len(ch["q"]) - 1).tobytes()),
        dict(name="P123_sparse_dim", type=h5_spec.dt_int(8, False), n=1, data=np.uint64(n).tobytes()),
        dict(name="p boundaries", type=bt, n=len(ch["p"]), data=bounds(ch["p"]), chunk=10, type_size=16,
             attrs=[("CLASS", "TABLE"), ("VERSION", "3.0"), ("TITLE", "Info p boundaries")], split=split),
        dict(name="q boundaries", type=bt, n=len(ch["q"]), data=bounds(ch["q"]), chunk=10, type_size=16),
        dict(name="pw channels", type=pt, n=len(pwt), data=bytes(pw_bytes), chunk=10, type_size=40,
             attrs=[("CLASS", "TABLE"), ("TITLE", "Partial wave info")], split=split),
        dict(name="row indices", type=h5_spec.dt_int(), n=n, data=np.asarray(ch["row"], "<i4").tobytes()),
        dict(name="column indices", type=h5_spec.dt_int(), n=n, data=np.asarray(ch["col"], "<i4").tobytes()),
        dict(name="values", type=h5_spec.dt_f64(), n=n, data=np.asarray(ch["val"], "<f8").tobytes()),
    ]
    h5_spec.write(path, ds, leaf_k=leaf_k)


@pytest.mark.parametrize("leaf_k,split", [(4, False), (2, False), (4, True)])
def test_reader_accepts_library_style_tables(tmp_path, leaf_k, split):
    ch = channel("lo_j1_J3_n8", 3)  # Nalpha > 10: the pw table spans several chunks
    assert len(np.asarray(ch["pwt"]).reshape(-1, 9)) > 10
    path = tmp_path / "lib.h5"
    _library_style_file(path, ch, leaf_k, split)
    f = h5_spec.File(path)  # the writer's own file parses
    assert f.datasets["pw channels"]["layout"]["class"] == "chunked"
    assert f.datasets["p boundaries"]["attrs"]["TITLE"] == "Info p boundaries"
    r, c, v = tt.read_P123_h5(path, ch["pw"], ch["p"], ch["q"])
    assert np.array_equal(r, ch["row"]) and np.array_equal(c, ch["col"]) and np.array_equal(v, ch["val"])


def test_file_name_is_the_references():
    ch = channel("lo_j1_J3_n8", 0)
    pwt = np.asarray(ch["pwt"]).reshape(-1, 9)
    name = tt.P123_h5_filename("Output", ch["pw"], len(ch["p"]) - 1, len(ch["q"]) - 1)
    J2, P = int(pwt[0][6]), int(pwt[0][8])
    assert name == f"Output/P123_sparse_JP_{J2}_{P}_Np_{len(ch['p']) - 1}_Nq_{len(ch['q']) - 1}_J2max_{ch['pw'].s.J_2N_max}.h5"


@pytest.mark.gpu
def test_run_handle_stores_and_loads_P123(tmp_path):
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=8, Nq_WP=8, Nphi=20, Nx=20,
                lab_energies="12", P123_folder=str(tmp_path))
    run = tt.Run(**opts)
    nnzs = []
    for c in range(run.num_channels):
        nnz = run.build_P123(c)
        nnzs.append(nnz)
        rowptr, col, val = run.P123_csr(c, nnz)
        run.store_P123_h5(c)
        pwt = run.host_array(0, c).reshape(-1, 9)
        pw = tt.PW(pwt, J_2N_max=1)
        p, q = run.host_array(1), run.host_array(2)
        path = tt.P123_h5_filename(str(tmp_path), pw, len(p) - 1, len(q) - 1)
        r, cc, v = tt.read_P123_h5(path, pw, p, q)
        rows = np.repeat(np.arange(len(rowptr) - 1, dtype=np.int32), np.diff(rowptr))
        assert np.array_equal(r, rows) and np.array_equal(cc, col) and np.array_equal(v, val)
        f = h5_spec.File(path)
        assert int(f.datasets["P123_sparse_dim"]["data"][0]) == nnz
    # a second run reads the files instead of building P123 (calculate_and_store_P123 = false)
    # and solves to the same U
    run2 = tt.Run(**opts)
    for c in range(run.num_channels):
        assert run2.load_P123_h5(c) == nnzs[c]
        rp2, col2, val2 = run2.P123_csr(c, nnzs[c])
        rp1, col1, val1 = run.P123_csr(c, nnzs[c])
        assert np.array_equal(rp1, rp2) and np.array_equal(col1, col2) and np.array_equal(val1, val2)
        U1, _ = run.solve(c, tt.PRECISION_FP64)
        U2, _ = run2.solve(c, tt.PRECISION_FP64)
        assert np.array_equal(U1, U2)
    with pytest.raises(tt.TicTacError):
        run2.load_P123_h5(0, str(tmp_path / "missing.h5"))
    run2.close()
    # calculate_and_store_P123 = false: build_P123 reads the files, as the reference does
    run3 = tt.Run(calculate_and_store_P123="false", **opts)
    for c in range(run.num_channels):
        assert run3.build_P123(c) == nnzs[c]
        assert np.array_equal(run3.solve(c, tt.PRECISION_FP64)[0], run.solve(c, tt.PRECISION_FP64)[0])
    run3.close()
    run4 = tt.Run(calculate_and_store_P123="false", **dict(opts, P123_folder=str(tmp_path / "none")))
    with pytest.raises(tt.TicTacError):
        run4.build_P123(0)
    run4.close()
    run.close()
