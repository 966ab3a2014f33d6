"""ctypes binding of the tictac_b200 C-ABI (include/tictac_b200.h).

The library is the in-tree build ``tic-tac_b200/lib/libtictac_b200.so``; there
is no Python or CPU implementation of the path behind this module.  Every call
raises ``TicTacError`` when the library returns a non-zero status.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, byref, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libtictac_b200.so"))

TT_OK = 0
TT_ERR_BADARG = 1
TT_ERR_NOMEM = 2
TT_ERR_CUDA = 3
TT_ERR_NOCONVERGE = 4
TT_ERR_IO = 5
TT_ERR_UNSUPPORTED = 6
TT_ERR_SINGULAR = 7

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_MIXED_SIMT = 2
PRECISION_PADE = 3

EXPORTED_SYMBOLS = (
    "tt_run_params_default", "tt_fill_P123_arrays", "tt_calculate_resolvent_array_in_SWP_basis",
    "tt_solve_faddeev_equations", "tt_free", "tt_last_error_string", "tt_device_count", "tt_run_create",
    "tt_run_destroy", "tt_run_num_channels", "tt_run_channel_info", "tt_run_num_energies", "tt_run_energies",
    "tt_run_E_bound", "tt_run_build_P123", "tt_run_build_A", "tt_run_build_resolvent", "tt_run_solve",
    "tt_run_release_channel", "tt_run_get_P123_csr", "tt_run_get_A", "tt_run_get_G", "tt_run_get_host_array",
    "tt_run_write_U_table", "tt_run_release_A", "tt_run_timer_start", "tt_run_timer_stop", "tt_kernel_launches",
    "tt_wigner_3j", "tt_wigner_6j", "tt_wigner_9j", "tt_clebsch_gordan", "tt_legendre_spharm_array",
    "tt_gauss_legendre", "tt_calculate_resolvent_array_in_SWP_basis_noalloc", "tt_profile_begin", "tt_profile_end",
    "tt_profile_read", "tt_solve_faddeev_adjoint", "tt_run_solve_adjoint", "tt_run_num_lecs", "tt_run_lec_derivative",
    "tt_store_P123_h5", "tt_read_P123_h5", "tt_P123_h5_filename", "tt_run_store_P123_h5", "tt_run_load_P123_h5",
    "tt_run_solve_energies", "tt_profile_select", "tt_run_adjoint_forward", "tt_run_adjoint_backward",
    "tt_run_swp_derivative", "tt_run_set_solve_option", "tt_release_cached_device_memory",
    "tt_cached_device_memory", "tt_solve_faddeev_equations_breakup", "tt_run_breakup_cells", "tt_run_solve_breakup",
    "tt_run_write_U_BU_table",
)

PROFILE_CLASSES = ("tc_update", "subpanel", "trsv", "residual", "a_build", "panel_trsm", "operands", "laswp", "form_L",
                   "subst_prep", "simt_update", "tc_panel", "fp64_update", "vector")


class TicTacError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tictac_b200 error {code}: {msg}")
        self.code = code


class tt_pw_states(ctypes.Structure):
    _fields_ = [("Nalpha", c_int), ("J_2N_max", c_int)] + [
        (f, POINTER(c_int)) for f in ("L_2N_array", "S_2N_array", "J_2N_array", "T_2N_array", "L_1N_array",
                                      "two_J_1N_array", "two_J_3N_array", "two_T_3N_array", "P_3N_array")]


class tt_fwp_states(ctypes.Structure):
    _fields_ = [("Np_WP", c_int), ("Nq_WP", c_int), ("p_WP_array", POINTER(c_double)),
                ("q_WP_array", POINTER(c_double))]


class tt_swp_states(ctypes.Structure):
    _fields_ = [("Np_WP", c_int), ("Nq_WP", c_int), ("num_2N_unco_states", c_int), ("num_2N_coup_states", c_int),
                ("E_bound", c_double)] + [
        (f, POINTER(c_double)) for f in ("e_SWP_unco_array", "e_SWP_coup_array", "C_SWP_unco_array",
                                         "C_SWP_coup_array", "q_WP_array")]


class tt_os_indexing(ctypes.Structure):
    _fields_ = [("num_T_lab", c_int), ("q_com_idx_array", POINTER(c_int)), ("deuteron_idx_array", POINTER(c_int)),
                ("num_deuteron_states", c_int)]


class tt_bu_indexing(ctypes.Structure):
    _fields_ = [("num_BU_chns", c_int), ("q_com_BU_idx_array", POINTER(c_int)), ("alphapq_idx_array", POINTER(c_int))]


class tt_run_params(ctypes.Structure):
    _fields_ = [("Nphi", c_int), ("Nx", c_int), ("tensor_force", c_int), ("isospin_breaking_1S0", c_int),
                ("production_run", c_int), ("precision", c_int), ("refine_tol", c_double),
                ("refine_max_iter", c_int)]


class tt_solve_report(ctypes.Structure):
    _fields_ = [("ms_A", c_double), ("ms_form", c_double), ("ms_factor", c_double), ("ms_solve", c_double),
                ("ms_refine", c_double), ("refine_iters", c_int), ("final_correction", c_double), ("info", c_int),
                ("ms_adjoint", c_double), ("adjoint_refine_iters", c_int), ("product_fallbacks", c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(path: str = LIB_PATH):
    """Load the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise TicTacError(TT_ERR_UNSUPPORTED, f"{path} is missing: run __graft_entry__.build() first")
    lib = ctypes.CDLL(path)
    lib.tt_last_error_string.restype = c_char_p
    lib.tt_run_destroy.restype = None
    lib.tt_free.restype = None
    lib.tt_run_params_default.restype = None
    lib.tt_kernel_launches.restype = ctypes.c_ulonglong
    for f in ("tt_wigner_3j", "tt_wigner_6j", "tt_wigner_9j", "tt_clebsch_gordan"):
        getattr(lib, f).restype = c_double
    _lib = lib
    return lib


def _check(rc):
    if rc != TT_OK:
        raise TicTacError(rc, _lib.tt_last_error_string().decode(errors="replace"))


def _iptr(a):
    return a.ctypes.data_as(POINTER(c_int))


def _dptr(a):
    return a.ctypes.data_as(POINTER(c_double))


def device_count() -> int:
    lib = load()
    n = c_int(0)
    rc = lib.tt_device_count(byref(n))
    return n.value if rc == TT_OK else 0


def cached_device_memory() -> int:
    """Bytes of released device blocks the library holds for reuse on the current device."""
    v = c_size_t()
    _check(load().tt_cached_device_memory(byref(v)))
    return v.value


def release_cached_device_memory() -> None:
    _check(load().tt_release_cached_device_memory())


def kernel_launches() -> int:
    return int(load().tt_kernel_launches())


def wigner3j(*a):
    return load().tt_wigner_3j(*[int(x) for x in a])


def wigner6j(*a):
    return load().tt_wigner_6j(*[int(x) for x in a])


def wigner9j(*a):
    return load().tt_wigner_9j(*[int(x) for x in a])


def clebsch_gordan(*a):
    return load().tt_clebsch_gordan(*[int(x) for x in a])


def spharm_array(lmax, x):
    out = np.zeros((lmax + 1) * (lmax + 2) // 2)
    _check(load().tt_legendre_spharm_array(int(lmax), c_double(x), _dptr(out)))
    return out


def gauss_legendre(n):
    x = np.zeros(n)
    w = np.zeros(n)
    _check(load().tt_gauss_legendre(int(n), _dptr(x), _dptr(w)))
    return x, w


def run_params(**kw) -> tt_run_params:
    lib = load()
    rp = tt_run_params()
    lib.tt_run_params_default(byref(rp))
    for k, v in kw.items():
        setattr(rp, k, v)
    return rp


class PW:
    """One channel's partial-wave table (9 ints per alpha: L S J T l 2j 2J 2T P)."""

    def __init__(self, table: np.ndarray, J_2N_max: int = 1):
        t = np.ascontiguousarray(np.asarray(table, dtype=np.int32).reshape(-1, 9))
        self._cols = [np.ascontiguousarray(t[:, k]) for k in range(9)]
        self.s = tt_pw_states(t.shape[0], J_2N_max, *[_iptr(c) for c in self._cols])
        self.Nalpha = t.shape[0]


def fill_P123_arrays(pw: PW, p_WP, q_WP, production_run=True, **rp_kw):
    """tt_fill_P123_arrays: row-major COO (row, col, val) of P123 built on the GPU."""
    lib = load()
    p = np.ascontiguousarray(p_WP, dtype=np.float64)
    q = np.ascontiguousarray(q_WP, dtype=np.float64)
    fwp = tt_fwp_states(len(p) - 1, len(q) - 1, _dptr(p), _dptr(q))
    rp = run_params(**rp_kw)
    val = POINTER(c_double)()
    row = POINTER(c_int)()
    col = POINTER(c_int)()
    nnz = c_size_t(0)
    _check(lib.tt_fill_P123_arrays(byref(val), byref(row), byref(col), byref(nnz), int(production_run), byref(fwp),
                                   byref(pw.s), byref(rp)))
    m = nnz.value
    try:
        v = np.ctypeslib.as_array(val, shape=(max(m, 1),))[:m].copy()
        r = np.ctypeslib.as_array(row, shape=(max(m, 1),))[:m].copy()
        c = np.ctypeslib.as_array(col, shape=(max(m, 1),))[:m].copy()
    finally:
        lib.tt_free(ctypes.cast(val, c_void_p))
        lib.tt_free(ctypes.cast(row, c_void_p))
        lib.tt_free(ctypes.cast(col, c_void_p))
    return r, c, v


def store_P123_h5(path, row, col, val, pw: PW, p_WP, q_WP) -> None:
    """tt_store_P123_h5: one channel's COO P123 in the reference's HDF5 layout."""
    lib = load()
    p = np.ascontiguousarray(p_WP, dtype=np.float64)
    q = np.ascontiguousarray(q_WP, dtype=np.float64)
    fwp = tt_fwp_states(len(p) - 1, len(q) - 1, _dptr(p), _dptr(q))
    r = np.ascontiguousarray(row, dtype=np.int32)
    c = np.ascontiguousarray(col, dtype=np.int32)
    v = np.ascontiguousarray(val, dtype=np.float64)
    if not (len(r) == len(c) == len(v)):
        raise ValueError("row, col and val must have the same length")
    _check(lib.tt_store_P123_h5(os.fsencode(path), _dptr(v), _iptr(r), _iptr(c), c_size_t(len(v)), byref(fwp),
                                byref(pw.s)))


def read_P123_h5(path, pw: PW, p_WP, q_WP):
    """tt_read_P123_h5: (row, col, val) of a P123 file after the reference's
    state-space checks against pw and the boundaries."""
    lib = load()
    p = np.ascontiguousarray(p_WP, dtype=np.float64)
    q = np.ascontiguousarray(q_WP, dtype=np.float64)
    fwp = tt_fwp_states(len(p) - 1, len(q) - 1, _dptr(p), _dptr(q))
    val = POINTER(c_double)()
    row = POINTER(c_int)()
    col = POINTER(c_int)()
    nnz = c_size_t(0)
    _check(lib.tt_read_P123_h5(os.fsencode(path), byref(val), byref(row), byref(col), byref(nnz), byref(fwp),
                               byref(pw.s)))
    m = nnz.value
    try:
        v = np.ctypeslib.as_array(val, shape=(max(m, 1),))[:m].copy()
        r = np.ctypeslib.as_array(row, shape=(max(m, 1),))[:m].copy()
        c = np.ctypeslib.as_array(col, shape=(max(m, 1),))[:m].copy()
    finally:
        lib.tt_free(ctypes.cast(val, c_void_p))
        lib.tt_free(ctypes.cast(row, c_void_p))
        lib.tt_free(ctypes.cast(col, c_void_p))
    return r, c, v


def P123_h5_filename(folder, pw: PW, Np_WP, Nq_WP) -> str:
    lib = load()
    buf = ctypes.create_string_buffer(4096)
    _check(lib.tt_P123_h5_filename(buf, c_size_t(len(buf)), os.fsencode(folder), byref(pw.s), Np_WP, Nq_WP))
    return buf.value.decode()


class SWP:
    def __init__(self, Np, Nq, n_unco, n_coup, E_bound, e_unco, e_coup, C_unco, C_coup, q_WP):
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else np.zeros(1)
                      for a in (e_unco, e_coup, C_unco, C_coup, q_WP)]
        self.s = tt_swp_states(Np, Nq, n_unco, n_coup, E_bound, *[_dptr(a) for a in self._keep])


def resolvent(G_E: float, swp: SWP, pw: PW, **rp_kw) -> np.ndarray:
    lib = load()
    n = pw.Nalpha * swp.s.Np_WP * swp.s.Nq_WP
    G = np.zeros(n, dtype=np.complex128)
    rp = run_params(**rp_kw)
    _check(lib.tt_calculate_resolvent_array_in_SWP_basis(G.ctypes.data_as(c_void_p), c_double(G_E), byref(swp.s),
                                                         byref(pw.s), byref(rp)))
    return G


class tt_kernel_profile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_ulonglong), ("ms", c_double), ("flops", c_double), ("bytes", c_double)]


def profile_begin(classes=None) -> None:
    """Start event timing of the kernel classes in PROFILE_CLASSES (or only of
    the named ones)."""
    lib = load()
    mask = (1 << len(PROFILE_CLASSES)) - 1 if classes is None else \
        sum(1 << PROFILE_CLASSES.index(c) for c in classes)
    lib.tt_profile_select.argtypes = [ctypes.c_ulonglong]
    _check(lib.tt_profile_select(mask))
    _check(lib.tt_profile_begin())


def profile_end() -> dict:
    """Stop timing; {class: {launches, ms, flops, bytes}} over the region."""
    lib = load()
    _check(lib.tt_profile_end())
    out = {}
    for i, name in enumerate(PROFILE_CLASSES):
        p = tt_kernel_profile()
        _check(lib.tt_profile_read(i, byref(p)))
        out[name] = {"launches": int(p.launches), "ms": p.ms, "flops": p.flops, "bytes": p.bytes}
    return out


def resolvent_noalloc(G_dev_ptr: int, energies, swp: SWP, pw: PW, stream: int = 0, **rp_kw) -> None:
    """tt_calculate_resolvent_array_in_SWP_basis_noalloc: resolvents of all
    `energies` into the caller's device buffer at address G_dev_ptr
    (complex128 [nE][n]), queued on `stream` (a cudaStream_t handle)."""
    lib = load()
    E = np.ascontiguousarray(energies, dtype=np.float64)
    rp = run_params(**rp_kw)
    _check(lib.tt_calculate_resolvent_array_in_SWP_basis_noalloc(
        c_void_p(G_dev_ptr), E.ctypes.data_as(c_void_p), ctypes.c_int(len(E)), byref(swp.s), byref(pw.s), byref(rp),
        c_void_p(stream)))


def solve_faddeev(G, P_val, P_row, P_colptr, V_unco, V_coup, swp: SWP, q_idx, deut, pw: PW, precision=PRECISION_MIXED,
                  **rp_kw):
    """tt_solve_faddeev_equations with the reference's CSC P123 and host arrays."""
    lib = load()
    G = np.ascontiguousarray(G, dtype=np.complex128)
    Pv = np.ascontiguousarray(P_val, dtype=np.float64)
    Pr = np.ascontiguousarray(P_row, dtype=np.int32)
    Pc = np.ascontiguousarray(P_colptr, dtype=np.uint64)
    Vu = np.ascontiguousarray(V_unco, dtype=np.float64)
    Vc = np.ascontiguousarray(V_coup if V_coup is not None and len(V_coup) else np.zeros(1), dtype=np.float64)
    qi = np.ascontiguousarray(q_idx, dtype=np.int32)
    di = np.ascontiguousarray(deut, dtype=np.int32)
    os_ = tt_os_indexing(len(qi), _iptr(qi), _iptr(di), len(di))
    rp = run_params(precision=precision, **rp_kw)
    U = np.zeros(len(qi) * len(di) * len(di), dtype=np.complex128)
    rep = tt_solve_report()
    _check(lib.tt_solve_faddeev_equations(U.ctypes.data_as(c_void_p), G.ctypes.data_as(c_void_p), _dptr(Pv),
                                          _iptr(Pr), Pc.ctypes.data_as(POINTER(c_size_t)), c_size_t(len(Pv)),
                                          _dptr(Vu), _dptr(Vc), byref(swp.s), byref(os_), byref(pw.s), byref(rp),
                                          byref(rep)))
    return U, rep.as_dict()


def solve_faddeev_breakup(G, P_val, P_row, P_colptr, V_unco, V_coup, swp: SWP, q_idx, deut, pw: PW, bu_start, bu_cells,
                          **rp_kw):
    """tt_solve_faddeev_equations_breakup (the Pade path): the elastic U and the
    breakup U_BU[d * num_cells + b] of the cells bu_cells[num][3] = (alpha, q, p),
    bu_start[nE + 1] their offsets per energy."""
    lib = load()
    G = np.ascontiguousarray(G, dtype=np.complex128)
    Pv = np.ascontiguousarray(P_val, dtype=np.float64)
    Pr = np.ascontiguousarray(P_row, dtype=np.int32)
    Pc = np.ascontiguousarray(P_colptr, dtype=np.uint64)
    Vu = np.ascontiguousarray(V_unco, dtype=np.float64)
    Vc = np.ascontiguousarray(V_coup if V_coup is not None and len(V_coup) else np.zeros(1), dtype=np.float64)
    qi = np.ascontiguousarray(q_idx, dtype=np.int32)
    di = np.ascontiguousarray(deut, dtype=np.int32)
    st = np.ascontiguousarray(bu_start, dtype=np.int32)
    cl = np.ascontiguousarray(np.asarray(bu_cells).reshape(-1), dtype=np.int32)
    num = cl.size // 3
    cl_buf = cl if cl.size else np.zeros(1, dtype=np.int32)
    os_ = tt_os_indexing(len(qi), _iptr(qi), _iptr(di), len(di))
    bu = tt_bu_indexing(num, _iptr(st), _iptr(cl_buf))
    rp = run_params(precision=PRECISION_PADE, **rp_kw)
    U = np.zeros(max(len(qi) * len(di) * len(di), 1), dtype=np.complex128)
    U_BU = np.zeros(max(len(di) * num, 1), dtype=np.complex128)
    rep = tt_solve_report()
    _check(lib.tt_solve_faddeev_equations_breakup(
        U.ctypes.data_as(c_void_p), U_BU.ctypes.data_as(c_void_p), byref(bu), G.ctypes.data_as(c_void_p), _dptr(Pv),
        _iptr(Pr), Pc.ctypes.data_as(POINTER(c_size_t)), c_size_t(len(Pv)), _dptr(Vu), _dptr(Vc), byref(swp.s),
        byref(os_), byref(pw.s), byref(rp), byref(rep)))
    return U[:len(qi) * len(di) * len(di)], U_BU[:len(di) * num], rep.as_dict()


def solve_faddeev_adjoint(G, P_val, P_row, P_colptr, V_unco, V_coup, swp: SWP, q_idx, deut, pw: PW, dV_unco, dV_coup,
                          precision=PRECISION_MIXED, **rp_kw):
    """tt_solve_faddeev_adjoint: U and dU/dtheta_k for the potential derivatives
    dV_unco [n_theta][...], dV_coup [n_theta][...] (layout of V_unco / V_coup),
    with the wave-packet basis and the resolvent held fixed.  Returns U,
    dU [n_theta][nE*nd*nd] and the solve report."""
    lib = load()
    G = np.ascontiguousarray(G, dtype=np.complex128)
    Pv = np.ascontiguousarray(P_val, dtype=np.float64)
    Pr = np.ascontiguousarray(P_row, dtype=np.int32)
    Pc = np.ascontiguousarray(P_colptr, dtype=np.uint64)
    Vu = np.ascontiguousarray(V_unco, dtype=np.float64)
    Vc = np.ascontiguousarray(V_coup if V_coup is not None and len(V_coup) else np.zeros(1), dtype=np.float64)
    dVu = np.ascontiguousarray(dV_unco, dtype=np.float64)
    n_theta = dVu.shape[0]
    dVc = np.ascontiguousarray(dV_coup if dV_coup is not None and np.size(dV_coup) else np.zeros((n_theta, 1)),
                               dtype=np.float64)
    qi = np.ascontiguousarray(q_idx, dtype=np.int32)
    di = np.ascontiguousarray(deut, dtype=np.int32)
    os_ = tt_os_indexing(len(qi), _iptr(qi), _iptr(di), len(di))
    rp = run_params(precision=precision, **rp_kw)
    U = np.zeros(len(qi) * len(di) * len(di), dtype=np.complex128)
    dU = np.zeros((n_theta, U.size), dtype=np.complex128)
    rep = tt_solve_report()
    _check(lib.tt_solve_faddeev_adjoint(U.ctypes.data_as(c_void_p), dU.ctypes.data_as(c_void_p), ctypes.c_int(n_theta),
                                        _dptr(dVu), _dptr(dVc), G.ctypes.data_as(c_void_p), _dptr(Pv), _iptr(Pr),
                                        Pc.ctypes.data_as(POINTER(c_size_t)), c_size_t(len(Pv)), _dptr(Vu), _dptr(Vc),
                                        byref(swp.s), byref(os_), byref(pw.s), byref(rp), byref(rep)))
    return U, dU, rep.as_dict()


class Run:
    """A configured run (tt_run_*): host state-space setup from key=value options
    (keywords) and input-list files (positional paths ending in .txt, applied
    first)."""

    def __init__(self, *input_lists, **opts):
        lib = load()
        args = [os.fspath(p) for p in input_lists] + [f"{k}={v}" for k, v in opts.items()]
        arr = (c_char_p * len(args))(*[a.encode() for a in args])
        self._h = c_void_p()
        _check(lib.tt_run_create(byref(self._h), len(args), arr))
        self.lib = lib

    def close(self):
        if self._h:
            self.lib.tt_run_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_channels(self):
        n = c_int()
        _check(self.lib.tt_run_num_channels(self._h, byref(n)))
        return n.value

    def channel_info(self, chn):
        v = [c_int() for _ in range(5)]
        _check(self.lib.tt_run_channel_info(self._h, chn, *[byref(x) for x in v]))
        return dict(zip(("Nalpha", "n", "two_J_3N", "P_3N", "n_deuteron"), [x.value for x in v]))

    def energies(self):
        nE = c_int()
        _check(self.lib.tt_run_num_energies(self._h, byref(nE)))
        T = np.zeros(nE.value)
        E = np.zeros(nE.value)
        q = np.zeros(nE.value, dtype=np.int32)
        _check(self.lib.tt_run_energies(self._h, _dptr(T), _dptr(E), _iptr(q)))
        return T, E, q

    @property
    def E_bound(self):
        e = c_double()
        _check(self.lib.tt_run_E_bound(self._h, byref(e)))
        return e.value

    def host_array(self, which, chn=0):
        dtype = np.int32 if which == 0 else np.float64
        cnt = c_size_t()
        _check(self.lib.tt_run_get_host_array(self._h, chn, which, None, byref(cnt)))
        out = np.zeros(cnt.value, dtype=dtype)
        _check(self.lib.tt_run_get_host_array(self._h, chn, which, out.ctypes.data_as(c_void_p), byref(cnt)))
        return out

    def build_P123(self, chn):
        nnz = c_int64()
        _check(self.lib.tt_run_build_P123(self._h, chn, byref(nnz)))
        return nnz.value

    def P123_csr(self, chn, nnz):
        n = self.channel_info(chn)["n"]
        rowptr = np.zeros(n + 1, dtype=np.int64)
        col = np.zeros(max(nnz, 1), dtype=np.int32)
        val = np.zeros(max(nnz, 1), dtype=np.float64)
        _check(self.lib.tt_run_get_P123_csr(self._h, chn, rowptr.ctypes.data_as(c_void_p), col.ctypes.data_as(c_void_p),
                                            val.ctypes.data_as(c_void_p)))
        return rowptr, col[:nnz], val[:nnz]

    def build_A(self, chn):
        ms = c_double()
        _check(self.lib.tt_run_build_A(self._h, chn, byref(ms)))
        return ms.value

    def A(self, chn):
        n = self.channel_info(chn)["n"]
        out = np.zeros((n, n))
        _check(self.lib.tt_run_get_A(self._h, chn, _dptr(out)))
        return out

    def build_resolvent(self, chn):
        _check(self.lib.tt_run_build_resolvent(self._h, chn))

    def G(self, chn):
        n = self.channel_info(chn)["n"]
        nE = len(self.energies()[0])
        out = np.zeros(n * nE, dtype=np.complex128)
        _check(self.lib.tt_run_get_G(self._h, chn, out.ctypes.data_as(c_void_p)))
        return out.reshape(nE, n)

    def solve(self, chn, precision=PRECISION_MIXED):
        info = self.channel_info(chn)
        nE = len(self.energies()[0])
        nd = info["n_deuteron"]
        U = np.zeros(nE * nd * nd, dtype=np.complex128)
        rep = tt_solve_report()
        _check(self.lib.tt_run_solve(self._h, chn, precision, U.ctypes.data_as(c_void_p), byref(rep)))
        return U, rep.as_dict()

    def solve_energies(self, chn, energy_idx, precision=PRECISION_MIXED):
        """tt_run_solve_energies: U of the selected on-shell energies, [d'][d][s] flattened."""
        idx = np.ascontiguousarray(energy_idx, dtype=np.int32)
        nd = self.channel_info(chn)["n_deuteron"]
        U = np.zeros(len(idx) * nd * nd, dtype=np.complex128)
        rep = tt_solve_report()
        _check(self.lib.tt_run_solve_energies(self._h, chn, precision, len(idx), _iptr(idx) if len(idx) else None,
                                              U.ctypes.data_as(c_void_p), byref(rep)))
        return U, rep.as_dict()

    def solve_adjoint(self, chn, dV_unco, dV_coup, precision=PRECISION_MIXED):
        """U and dU/dtheta_k for potential derivatives over all 2N channels of the
        run ([n_theta][...] in the layout of host_array(3) / host_array(4)): the
        total derivative (the SWP basis, deuteron energy and resolvent move with
        the potential), or with them held fixed when the run has
        adjoint_basis=fixed."""
        info = self.channel_info(chn)
        nE = len(self.energies()[0])
        nd = info["n_deuteron"]
        dVu = np.ascontiguousarray(dV_unco, dtype=np.float64)
        n_theta = dVu.shape[0]
        dVc = np.ascontiguousarray(dV_coup if dV_coup is not None and np.size(dV_coup) else np.zeros((n_theta, 1)),
                                   dtype=np.float64)
        U = np.zeros(nE * nd * nd, dtype=np.complex128)
        dU = np.zeros((n_theta, U.size), dtype=np.complex128)
        rep = tt_solve_report()
        _check(self.lib.tt_run_solve_adjoint(self._h, chn, precision, ctypes.c_int(n_theta), _dptr(dVu), _dptr(dVc),
                                             U.ctypes.data_as(c_void_p), dU.ctypes.data_as(c_void_p), byref(rep)))
        return U, dU, rep.as_dict()

    def adjoint_forward(self, chn, precision=PRECISION_MIXED):
        """tt_run_adjoint_forward: U, keeping the factors for adjoint_backward."""
        info = self.channel_info(chn)
        nE = len(self.energies()[0])
        nd = info["n_deuteron"]
        U = np.zeros(nE * nd * nd, dtype=np.complex128)
        rep = tt_solve_report()
        _check(self.lib.tt_run_adjoint_forward(self._h, chn, precision, U.ctypes.data_as(c_void_p), byref(rep)))
        return U, rep.as_dict()

    def adjoint_backward(self, chn, dV_unco, dV_coup, U_bar):
        """tt_run_adjoint_backward: theta_bar_k = Re sum conj(U_bar) dU/dtheta_k."""
        dVu = np.ascontiguousarray(dV_unco, dtype=np.float64)
        n_theta = dVu.shape[0]
        dVc = np.ascontiguousarray(dV_coup if dV_coup is not None and np.size(dV_coup) else np.zeros((n_theta, 1)),
                                   dtype=np.float64)
        Ub = np.ascontiguousarray(U_bar, dtype=np.complex128)
        out = np.zeros(n_theta, dtype=np.float64)
        rep = tt_solve_report()
        _check(self.lib.tt_run_adjoint_backward(self._h, chn, ctypes.c_int(n_theta), _dptr(dVu), _dptr(dVc),
                                                Ub.ctypes.data_as(c_void_p), _dptr(out), byref(rep)))
        return out, rep.as_dict()

    def swp_derivative(self, dV_unco, dV_coup):
        """tt_run_swp_derivative: (dC_unco, dC_coup, de_unco, de_coup, dE_bound)."""
        dVu = np.ascontiguousarray(dV_unco, dtype=np.float64)
        dVc = np.ascontiguousarray(dV_coup if dV_coup is not None and np.size(dV_coup) else np.zeros(1),
                                   dtype=np.float64)
        out = [np.zeros_like(self.host_array(w)) for w in (5, 6, 7, 8)]
        dEb = c_double(0)
        _check(self.lib.tt_run_swp_derivative(self._h, _dptr(dVu), _dptr(dVc), *[_dptr(o) if o.size else None
                                                                                  for o in out], byref(dEb)))
        return tuple(out) + (dEb.value,)

    def lecs(self):
        """Values of the potential's adjustable low-energy constants."""
        n = ctypes.c_int()
        _check(self.lib.tt_run_num_lecs(self._h, byref(n), None))
        v = np.zeros(max(1, n.value))
        _check(self.lib.tt_run_num_lecs(self._h, byref(n), _dptr(v)))
        return v[:n.value]

    def lec_derivative(self, k):
        """dV/dLEC_k in the WP basis for all 2N channels (uncoupled, coupled)."""
        dVu = np.zeros_like(self.host_array(3))
        dVc = np.zeros(max(1, self.host_array(4).size))
        _check(self.lib.tt_run_lec_derivative(self._h, k, _dptr(dVu), _dptr(dVc)))
        return dVu, dVc[:self.host_array(4).size]

    def set_solve_option(self, key, value):
        """Change a solve option (tc_product, panel_width, panel_order, inverse_block, cta_pairs, energy_batch,
        refine_tol, refine_max_iter) for the next solves."""
        _check(self.lib.tt_run_set_solve_option(self._h, str(key).encode(), str(value).encode()))

    def release(self, chn):
        _check(self.lib.tt_run_release_channel(self._h, chn))

    def release_A(self, chn):
        _check(self.lib.tt_run_release_A(self._h, chn))

    def timer_start(self):
        _check(self.lib.tt_run_timer_start(self._h))

    def timer_stop(self):
        ms = c_double()
        _check(self.lib.tt_run_timer_stop(self._h, byref(ms)))
        return ms.value

    def store_P123_h5(self, chn, path=None):
        """Writes the channel's resident P123 (after build_P123) in the reference's
        HDF5 layout; path None = the reference's name in the run's P123_folder."""
        _check(self.lib.tt_run_store_P123_h5(self._h, chn, None if path is None else os.fsencode(path)))

    def load_P123_h5(self, chn, path=None):
        """Makes a P123 file the channel's resident P123 (the reference's
        calculate_and_store_P123 = false path); returns nnz."""
        nnz = c_int64()
        _check(self.lib.tt_run_load_P123_h5(self._h, chn, None if path is None else os.fsencode(path), byref(nnz)))
        return nnz.value

    def write_U_table(self, chn, U, path):
        U = np.ascontiguousarray(U, dtype=np.complex128)
        _check(self.lib.tt_run_write_U_table(self._h, chn, U.ctypes.data_as(c_void_p), path.encode()))

    def breakup_cells(self, chn):
        """tt_run_breakup_cells: (start[nE + 1], cells[num][3] = (alpha, q bin, p bin))."""
        chn = int(chn)
        num = c_int()
        _check(self.lib.tt_run_breakup_cells(self._h, chn, byref(num), None, None))
        start = np.zeros(len(self.energies()[0]) + 1, dtype=np.int32)
        cells = np.zeros(max(3 * num.value, 1), dtype=np.int32)
        _check(self.lib.tt_run_breakup_cells(self._h, chn, byref(num), _iptr(start), _iptr(cells)))
        return start, cells[:3 * num.value].reshape(-1, 3)

    def solve_breakup(self, chn):
        """tt_run_solve_breakup: the Pade solve's elastic U and breakup U_BU[d * num_cells + b]."""
        chn = int(chn)
        nE = len(self.energies()[0])
        nd = self.channel_info(chn)["n_deuteron"]
        num = c_int()
        _check(self.lib.tt_run_breakup_cells(self._h, chn, byref(num), None, None))
        U = np.zeros(max(nE * nd * nd, 1), dtype=np.complex128)
        U_BU = np.zeros(max(nd * num.value, 1), dtype=np.complex128)
        rep = tt_solve_report()
        _check(self.lib.tt_run_solve_breakup(self._h, chn, U.ctypes.data_as(c_void_p), U_BU.ctypes.data_as(c_void_p),
                                             byref(rep)))
        return U[:nE * nd * nd], U_BU[:nd * num.value], rep.as_dict()

    def write_U_BU_table(self, chn, U_BU, path):
        U_BU = np.ascontiguousarray(U_BU, dtype=np.complex128)
        _check(self.lib.tt_run_write_U_BU_table(self._h, int(chn), U_BU.ctypes.data_as(c_void_p) if U_BU.size else None,
                                                os.fsencode(path)))
