"""ctypes binding of libop2b's C ABI (include/op2b.h).

The functions mirror the OP2 C/C++ API (op2/include/op_lib_c.h:75-121,
op_lib_cpp.h:127-203): same names, same argument meaning.  Python-side
conveniences: op_decl_dat takes a numpy array and derives type and size,
op_arg_gbl takes a numpy array (written back in place for INC/MIN/MAX, as the
reference writes back into the caller's variable), op_fetch_data returns a
new numpy array.  Errors raise Op2Error with the library's message.

The library must exist (build with op2b.build.build()); there is no fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

OP_READ, OP_WRITE, OP_RW, OP_INC, OP_MIN, OP_MAX, OP_WORK = range(7)
OP_ARG_GBL, OP_ARG_DAT, OP_ARG_IDX, OP_ARG_INFO = range(4)
OP_STAGE_NONE, OP_STAGE_INC, OP_STAGE_ALL, OP_STAGE_PERMUTE, OP_COLOR2 = range(5)
OP2B_INC_ATOMIC, OP2B_INC_COLOR, OP2B_INC_HYBRID, OP2B_INC_GATHER = range(4)
OP_ID = None
OP_GBL = None

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libop2b.so")


class Op2Error(RuntimeError):
    pass


class op_set_core(ctypes.Structure):
    _fields_ = [("index", ctypes.c_int), ("size", ctypes.c_int), ("name", ctypes.c_char_p),
                ("core_size", ctypes.c_int), ("exec_size", ctypes.c_int),
                ("nonexec_size", ctypes.c_int)]


class op_map_core(ctypes.Structure):
    pass


op_map_core._fields_ = [("index", ctypes.c_int), ("from_", ctypes.POINTER(op_set_core)),
                        ("to", ctypes.POINTER(op_set_core)), ("dim", ctypes.c_int),
                        ("map", ctypes.POINTER(ctypes.c_int)),
                        ("map_d", ctypes.POINTER(ctypes.c_int)), ("name", ctypes.c_char_p)]


class op_dat_core(ctypes.Structure):
    _fields_ = [("index", ctypes.c_int), ("set", ctypes.POINTER(op_set_core)),
                ("dim", ctypes.c_int), ("size", ctypes.c_int), ("data", ctypes.c_void_p),
                ("data_d", ctypes.c_void_p), ("type", ctypes.c_char_p), ("name", ctypes.c_char_p)]


op_set = ctypes.POINTER(op_set_core)
op_map = ctypes.POINTER(op_map_core)
op_dat = ctypes.POINTER(op_dat_core)


class op_arg(ctypes.Structure):
    _fields_ = [("index", ctypes.c_int), ("dat", op_dat), ("map", op_map),
                ("dim", ctypes.c_int), ("idx", ctypes.c_int), ("size", ctypes.c_int),
                ("data", ctypes.c_void_p), ("data_d", ctypes.c_void_p),
                ("map_data", ctypes.POINTER(ctypes.c_int)),
                ("map_data_d", ctypes.POINTER(ctypes.c_int)), ("type", ctypes.c_char_p),
                ("acc", ctypes.c_int), ("argtype", ctypes.c_int), ("sent", ctypes.c_int),
                ("opt", ctypes.c_int)]


# every exported symbol and its (restype, argtypes); the header lists the same set
_SIGS = {
    "op_init": (None, [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]),
    "op_exit": (None, []),
    "op_decl_set": (op_set, [ctypes.c_int, ctypes.c_char_p]),
    "op_decl_map": (op_map, [op_set, op_set, ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p]),
    "op_decl_dat_char": (op_dat, [op_set, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                  ctypes.c_void_p, ctypes.c_char_p]),
    "op_decl_dat_temp_char": (op_dat, [op_set, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                       ctypes.c_char_p]),
    "op_free_dat_temp_char": (ctypes.c_int, [op_dat]),
    "op_decl_dat_overlay": (op_dat, [op_set, op_dat]),
    "op_decl_dat_overlay_ptr": (op_dat, [op_set, ctypes.c_void_p]),
    "op_decl_const_char": (None, [ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_char_p]),
    "op_arg_dat": (op_arg, [op_dat, ctypes.c_int, op_map, ctypes.c_int, ctypes.c_char_p,
                            ctypes.c_int]),
    "op_opt_arg_dat": (op_arg, [ctypes.c_int, op_dat, ctypes.c_int, op_map, ctypes.c_int,
                                ctypes.c_char_p, ctypes.c_int]),
    "op_arg_gbl_char": (op_arg, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                 ctypes.c_int]),
    "op_opt_arg_gbl_char": (op_arg, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    "op_arg_info_char": (op_arg, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                  ctypes.c_int]),
    "op_arg_idx": (op_arg, [ctypes.c_int, op_map]),
    "op_par_loop_c": (ctypes.c_int, [ctypes.c_char_p, op_set, ctypes.c_int,
                                     ctypes.POINTER(op_arg)]),
    "op_par_loop_save_soln": (None, [ctypes.c_char_p, op_set] + [op_arg] * 2),
    "op_par_loop_adt_calc": (None, [ctypes.c_char_p, op_set] + [op_arg] * 6),
    "op_par_loop_res_calc": (None, [ctypes.c_char_p, op_set] + [op_arg] * 8),
    "op_par_loop_bres_calc": (None, [ctypes.c_char_p, op_set] + [op_arg] * 6),
    "op_par_loop_update": (None, [ctypes.c_char_p, op_set] + [op_arg] * 8),
    "op_fetch_data_char": (None, [op_dat, ctypes.c_void_p]),
    "op_fetch_data_idx_char": (None, [op_dat, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "op_print_dat_to_binfile": (None, [op_dat, ctypes.c_char_p]),
    "op_print_dat_to_txtfile": (None, [op_dat, ctypes.c_char_p]),
    "op_get_size": (ctypes.c_int, [op_set]),
    "op_timers": (None, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "op_timing_output": (None, []),
    "op_diagnostic_output": (None, []),
    "op_rank": (None, [ctypes.POINTER(ctypes.c_int)]),
    "op2b_last_error": (ctypes.c_char_p, []),
    "op2b_status": (ctypes.c_int, []),
    "op2b_dat_upload": (ctypes.c_int, [op_dat, ctypes.c_void_p, ctypes.c_size_t]),
    "op2b_dat_device_ptr": (ctypes.c_void_p, [op_dat]),
    "op2b_map_device_ptr": (ctypes.c_void_p, [op_map]),
    "op2b_set_option": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_long]),
    "op2b_register_kernel": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p]),
    "op2b_register_prelude": (ctypes.c_int, [ctypes.c_char_p]),
    "op2b_get_option": (ctypes.c_long, [ctypes.c_char_p]),
    "op2b_loop_stats": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_long),
                                       ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double)]),
    "op2b_reset_stats": (None, []),
    "op2b_kernel_launches": (ctypes.c_long, []),
    "op2b_set_stream": (ctypes.c_int, [ctypes.c_void_p]),
    "op2b_get_stream": (ctypes.c_void_p, []),
    "op2b_synchronize": (ctypes.c_int, []),
    "op2b_update_noalloc": (ctypes.c_int, [ctypes.c_int] + [ctypes.c_void_p] * 8),
    "op2b_dat_pack": (ctypes.c_int, [op_dat, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "op2b_dat_unpack": (ctypes.c_int, [op_dat, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p]),
    "op_profile_start": (None, [ctypes.c_char_p]),
    "op_profile_enter": (None, [ctypes.c_char_p]),
    "op_profile_enter_kernel": (None, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]),
    "op_profile_next": (None, [ctypes.c_char_p]),
    "op_profile_exit": (None, []),
    "op_profile_end": (None, []),
    "op_profile_output": (None, []),
    "op_profile_output_json": (None, [ctypes.c_char_p]),
    "op_decl_set_hdf5": (op_set, [ctypes.c_char_p, ctypes.c_char_p]),
    "op_decl_set_hdf5_infer_size": (op_set, [ctypes.c_char_p] * 3),
    "op_decl_map_hdf5": (op_map, [op_set, op_set, ctypes.c_int, ctypes.c_char_p,
                                  ctypes.c_char_p]),
    "op_decl_dat_hdf5": (op_dat, [op_set, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p,
                                  ctypes.c_char_p]),
    "op_get_const_hdf5": (None, [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                 ctypes.c_void_p, ctypes.c_char_p]),
    "op_dump_to_hdf5": (None, [ctypes.c_char_p]),
    "op_write_const_hdf5": (None, [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                   ctypes.c_void_p, ctypes.c_char_p]),
    "op_fetch_data_hdf5_file": (None, [op_dat, ctypes.c_char_p]),
    "op_fetch_data_hdf5_file_path": (None, [op_dat, ctypes.c_char_p, ctypes.c_char_p]),
    "op2b_h5_info": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_longlong), ctypes.c_char_p,
                                    ctypes.c_int]),
    "op2b_h5_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                    ctypes.c_void_p, ctypes.c_longlong]),
    "op2b_h5_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                     ctypes.c_int, ctypes.POINTER(ctypes.c_longlong),
                                     ctypes.c_void_p]),
    "op2b_h5_set_attr": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                        ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p]),
    "op2b_h5_get_attr": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                        ctypes.c_char_p, ctypes.c_int]),
    "op2b_h5_list": (ctypes.c_longlong, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_longlong]),
}


class op_plan(ctypes.Structure):
    """include/op2b_plan.h (field order of op2/include/op_rt_support.h:46-88)."""


_ip = ctypes.POINTER(ctypes.c_int)
op_plan._fields_ = [
    ("name", ctypes.c_char_p), ("set", op_set), ("nargs", ctypes.c_int), ("ninds", ctypes.c_int),
    ("ninds_staged", ctypes.c_int), ("part_size", ctypes.c_int),
    ("maps", ctypes.POINTER(op_map)), ("dats", ctypes.POINTER(op_dat)), ("idxs", _ip),
    ("optflags", _ip), ("accs", _ip), ("inds_staged", _ip),
    ("nthrcol", _ip), ("thrcol", _ip), ("col_reord", _ip), ("col_offsets", ctypes.POINTER(_ip)),
    ("color2_offsets", _ip), ("offset", _ip), ("offset_d", _ip), ("ind_map", _ip),
    ("ind_maps", ctypes.POINTER(_ip)), ("ind_offs", _ip), ("ind_sizes", _ip),
    ("nindirect", _ip), ("loc_map", ctypes.POINTER(ctypes.c_short)),
    ("loc_maps", ctypes.POINTER(ctypes.POINTER(ctypes.c_short))), ("nblocks", ctypes.c_int),
    ("nelems", _ip), ("nelems_d", _ip), ("ncolors_core", ctypes.c_int),
    ("ncolors_owned", ctypes.c_int), ("ncolors", ctypes.c_int), ("ncolblk", _ip),
    ("blkmap", _ip), ("blkmap_d", _ip), ("nsharedCol", _ip), ("nshared", ctypes.c_int),
    ("transfer", ctypes.c_float), ("transfer2", ctypes.c_float), ("count", ctypes.c_int)]

_SIGS.update({
    "op_plan_get_stage": (ctypes.POINTER(op_plan), [ctypes.c_char_p, op_set, ctypes.c_int,
                                                     ctypes.c_int, ctypes.POINTER(op_arg),
                                                     ctypes.c_int, _ip, ctypes.c_int]),
    "op_plan_get_stage_upload": (ctypes.POINTER(op_plan),
                                 [ctypes.c_char_p, op_set, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(op_arg), ctypes.c_int, _ip, ctypes.c_int,
                                  ctypes.c_int]),
    "op_plan_get": (ctypes.POINTER(op_plan), [ctypes.c_char_p, op_set, ctypes.c_int,
                                              ctypes.c_int, ctypes.POINTER(op_arg),
                                              ctypes.c_int, _ip]),
    "op_plan_check": (None, [op_plan, ctypes.c_int, _ip]),
    "op2b_plan_validate": (ctypes.c_int, [ctypes.POINTER(op_plan),
                                          ctypes.POINTER(ctypes.c_long)]),
    "op2b_plan_build_ms": (ctypes.c_double, [ctypes.POINTER(op_plan)]),
    "op2b_plan_device_blkmap": (ctypes.c_void_p, [ctypes.POINTER(op_plan)]),
    "op2b_plan_device_thrcol": (ctypes.c_void_p, [ctypes.POINTER(op_plan)]),
    "op2b_plan_release_all": (None, []),
    "op_renumber": (None, [op_map]),
    "op_renumber_ptr": (None, [ctypes.c_void_p]),
    "op2b_renumber": (ctypes.c_int, [op_map, ctypes.POINTER(ctypes.c_long)]),
    "op2b_set_permutation": (ctypes.c_int, [op_set, ctypes.c_void_p]),
})


def op_renumber(base, stats: bool = True):
    """Renumber the mesh from `base` (GPU reverse Cuthill-McKee); returns the
    base map's bandwidth (max, avg) before and after, or None with
    stats=False (as the C API's op_renumber, which does not measure them)."""
    st = (ctypes.c_long * 4)() if stats else None
    if load().op2b_renumber(base, st) != 0:
        _check(False, "op_renumber")
    if not stats:
        return None
    return dict(before_max=st[0], before_avg=st[1], after_max=st[2], after_avg=st[3])


def set_permutation(set_) -> np.ndarray:
    """perm[i] = current index of the element declared as i."""
    n = set_.contents.size
    out = np.zeros(max(n, 1), np.int32)
    if load().op2b_set_permutation(set_, out.ctypes.data) < 0:
        _check(False, "op2b_set_permutation")
    return out[:n]


def op_plan_get_stage(name: str, set_, part_size: int, args, inds, staging: int):
    arr = (op_arg * len(args))(*args)
    ind = (ctypes.c_int * len(inds))(*inds)
    p = load().op_plan_get_stage(_b(name), set_, int(part_size), len(args), arr, max(inds) + 1,
                                 ind, int(staging))
    if not p:
        _check(False, "op_plan_get_stage")
    return p


def plan_arrays(p) -> dict:
    """Host copies of a plan's arrays as numpy arrays (names of op_rt_support.h)."""
    o = p.contents
    nb, nst, ninds = o.nblocks, o.ninds_staged, o.ninds
    n = o.set.contents.size
    A = lambda ptr, cnt, dt=np.int32: np.ctypeslib.as_array(ptr, shape=(cnt,)).astype(dt).copy() \
        if cnt > 0 else np.zeros(0, dt)
    d = dict(nblocks=nb, ncolors=o.ncolors, ninds_staged=nst, nshared=o.nshared,
             transfer=o.transfer, transfer2=o.transfer2, count=o.count,
             nthrcol=A(o.nthrcol, nb), thrcol=A(o.thrcol, n), offset=A(o.offset, nb),
             nelems=A(o.nelems, nb), ind_offs=A(o.ind_offs, nb * nst),
             ind_sizes=A(o.ind_sizes, nb * nst), nindirect=A(o.nindirect, ninds),
             inds_staged=A(o.inds_staged, o.nargs))
    ncb = max(o.ncolors, 0)
    d["ncolblk"] = A(o.ncolblk, ncb if ncb else 0)
    d["blkmap"] = A(o.blkmap, nb)
    d["nsharedCol"] = A(o.nsharedCol, ncb)
    for m in range(nst):
        used = int(d["ind_sizes"][m::nst].sum()) if nb else 0
        d[f"ind_map{m}"] = A(o.ind_maps[m], used)
    for a in range(o.nargs):
        if o.loc_maps[a]:
            d[f"loc_map{a}"] = A(o.loc_maps[a], n, np.int16)
    if o.col_reord:
        d["col_reord"] = A(o.col_reord, n)
        tot = int((d["nthrcol"] + 1).sum())
        d["col_offsets"] = A(o.col_offsets[0], tot)
    return d


def plan_validate(p):
    det = (ctypes.c_long * 8)()
    n = load().op2b_plan_validate(p, det)
    if n < 0:
        _check(False, "op2b_plan_validate")
    return n, list(det)

_lib = None


def load(path: str | None = None):
    """Load libop2b.so (built in-tree).  Raises if it is missing: no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise Op2Error(f"{p} is missing: build it with `python op2-common_b200/op2b/build.py`")
    L = ctypes.CDLL(p)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols():
    return sorted(_SIGS)


def last_error() -> str:
    return load().op2b_last_error().decode(errors="replace")


def _check(ok: bool = True, what: str = ""):
    msg = last_error()
    if not ok:
        raise Op2Error(msg or what)


def _b(s):
    return None if s is None else s.encode()


_TYPES = {np.dtype(np.float64): "double", np.dtype(np.float32): "float",
          np.dtype(np.int32): "int"}

# arrays handed to the library whose lifetime must cover the call
_keep = []


def op_init(argv=(), diags: int = 0):
    L = load()
    arr = (ctypes.c_char_p * (len(argv) + 1))(*[_b(a) for a in argv], None)
    L.op_init(len(argv), arr, diags)
    if L.op2b_status() != 0:
        raise Op2Error("op_init failed: " + L.op2b_last_error().decode())


def op_exit():
    load().op_exit()
    _keep.clear()


def op_decl_set(size: int, name: str):
    s = load().op_decl_set(int(size), _b(name))
    if not s:
        _check(False, "op_decl_set")
    return s


def op_decl_map(frm, to, dim: int, data, name: str):
    a = np.ascontiguousarray(data, dtype=np.int32)
    m = load().op_decl_map(frm, to, int(dim), a.ctypes.data if a.size else None, _b(name))
    if not m:
        _check(False, "op_decl_map")
    return m


def op_decl_dat(set_, dim: int, type_: str | None, data, name: str):
    """op_decl_dat<T> (op_lib_cpp.h:127-137): the numpy dtype must match `type_`.
    data=None declares a zero-initialised dat (the reference callocs when it is
    given no data, op2/src/core/op_lib_core.cpp:520-537); nothing is uploaded."""
    if data is None:
        if type_ is None:
            raise Op2Error("op_decl_dat: needs data or a type")
        tb = {"double": 8, "float": 4, "int": 4}[type_.split(":")[0]]
        d = load().op_decl_dat_char(set_, int(dim), _b(type_), tb, None, _b(name))
    else:
        a = np.ascontiguousarray(data)
        t = _TYPES.get(a.dtype)
        if t is None or (type_ is not None and type_.split(":")[0] != t):
            raise Op2Error(f"incorrect type specified for dataset \"{name}\"")
        d = load().op_decl_dat_char(set_, int(dim), _b(type_ or t), a.dtype.itemsize,
                                    a.ctypes.data if a.size else None, _b(name))
    if not d:
        _check(False, "op_decl_dat")
    return d


def op_decl_dat_temp(set_, dim: int, type_: str, name: str):
    """op_decl_dat_temp<T> (op_lib_cpp.h): a zeroed dat, freed by op_free_dat_temp."""
    tb = {"double": 8, "float": 4, "int": 4}[type_.split(":")[0]]
    d = load().op_decl_dat_temp_char(set_, int(dim), _b(type_), tb, _b(name))
    if not d:
        _check(False, "op_decl_dat_temp")
    return d


def op_free_dat_temp(dat) -> int:
    return load().op_free_dat_temp_char(dat)


def op_decl_dat_overlay(set_, dat):
    """op_decl_dat_overlay (op_lib_c.h:85): `dat`'s storage seen as a dat on `set_`."""
    d = load().op_decl_dat_overlay(set_, dat)
    if not d:
        _check(False, "op_decl_dat_overlay")
    return d


def op_decl_dat_overlay_ptr(set_, data: np.ndarray):
    """op_decl_dat_overlay_ptr (op_lib_c.h:86): the dat declared from `data`."""
    d = load().op_decl_dat_overlay_ptr(set_, data.ctypes.data)
    if not d:
        _check(False, "op_decl_dat_overlay_ptr")
    return d


def op_decl_const(dim: int, type_: str, value, name: str):
    a = np.ascontiguousarray(np.atleast_1d(value),
                             dtype={"double": np.float64, "float": np.float32,
                                    "int": np.int32}[type_])
    load().op_decl_const_char(int(dim), _b(type_), a.dtype.itemsize, a.ctypes.data, _b(name))


def op_arg_dat(dat, idx: int, map_, dim: int, type_: str, acc: int):
    return load().op_arg_dat(dat, int(idx), map_, int(dim), _b(type_), int(acc))


def op_opt_arg_dat(opt: int, dat, idx: int, map_, dim: int, type_: str, acc: int):
    return load().op_opt_arg_dat(int(opt), dat, int(idx), map_, int(dim), _b(type_), int(acc))


def op_arg_gbl(data: np.ndarray, dim: int, type_: str, acc: int):
    if not isinstance(data, np.ndarray) or not data.flags.c_contiguous:
        raise Op2Error("op_arg_gbl: pass a contiguous numpy array (written back in place)")
    t = _TYPES.get(data.dtype)
    if t != type_:
        return load().op_arg_gbl_char(data.ctypes.data, int(dim), b"error", data.dtype.itemsize,
                                      int(acc))
    _keep.append(data)
    return load().op_arg_gbl_char(data.ctypes.data, int(dim), _b(type_), data.dtype.itemsize,
                                  int(acc))


def op_opt_arg_gbl(opt: int, data: np.ndarray, dim: int, type_: str, acc: int):
    if not isinstance(data, np.ndarray) or not data.flags.c_contiguous:
        raise Op2Error("op_opt_arg_gbl: pass a contiguous numpy array (written back in place)")
    _keep.append(data)
    return load().op_opt_arg_gbl_char(int(opt), data.ctypes.data, int(dim), _b(type_),
                                      data.dtype.itemsize, int(acc))


def op_arg_info(data: np.ndarray, dim: int, type_: str, ref: int):
    _keep.append(data)
    return load().op_arg_info_char(data.ctypes.data, int(dim), _b(type_), data.dtype.itemsize,
                                   int(ref))


def op_arg_idx(idx: int, map_):
    return load().op_arg_idx(int(idx), map_)


def op_par_loop(name: str, set_, *args):
    """op_par_loop(kernel, name, set, args...) without the host kernel pointer."""
    arr = (op_arg * len(args))(*args)
    rc = load().op_par_loop_c(_b(name), set_, len(args), arr)
    if len(_keep) > 64:
        del _keep[:-16]
    if rc != 0:
        _check(False, f"op_par_loop({name})")


def op_fetch_data(dat, out: np.ndarray | None = None) -> np.ndarray:
    """The dat's values (set size x dim) in a new array, or into `out` (a
    C-contiguous array of that shape and type, e.g. page-locked memory the
    caller keeps for its results)."""
    d = dat.contents
    t = d.type.decode().split(":")[0]
    dt = {"double": np.float64, "float": np.float32, "int": np.int32}[t]
    n = d.set.contents.size
    if out is None:
        out = np.empty((n, d.dim), dtype=dt)
    elif out.shape != (n, d.dim) or out.dtype != dt or not out.flags.c_contiguous:
        raise Op2Error(f"op_fetch_data: out must be a C-contiguous {np.dtype(dt)} array of "
                       f"shape {(n, d.dim)}")
    before = load().op2b_last_error()
    load().op_fetch_data_char(dat, out.ctypes.data)
    after = load().op2b_last_error()
    if after and after != before:
        raise Op2Error(after.decode())
    return out


def op_fetch_data_idx(dat, low: int, high: int) -> np.ndarray:
    d = dat.contents
    t = d.type.decode().split(":")[0]
    dt = {"double": np.float64, "float": np.float32, "int": np.int32}[t]
    out = np.empty((max(high - low + 1, 0), d.dim), dtype=dt)
    load().op_fetch_data_idx_char(dat, out.ctypes.data, int(low), int(high))
    return out


# ---- HDF5 mesh I/O (include/op_hdf5.h): the OP2 calls, then the host helpers

_H5_DTYPES = {"int": np.int32, "long": np.int64, "long long": np.int64, "float": np.float32,
              "double": np.float64}


def _fails(call):
    """Run `call`; raise Op2Error if it recorded a new error."""
    before = load().op2b_last_error()
    r = call()
    after = load().op2b_last_error()
    if after and after != before:
        raise Op2Error(after.decode())
    return r


def _declared(h, what: str):
    if not h:
        _check(False, what)
    return h


def op_decl_set_hdf5(file: str, name: str):
    return _declared(load().op_decl_set_hdf5(_b(file), _b(name)), "op_decl_set_hdf5")


def op_decl_set_hdf5_infer_size(file: str, name: str, set_dataset_name: str):
    return _declared(load().op_decl_set_hdf5_infer_size(_b(file), _b(name),
                                                        _b(set_dataset_name)),
                     "op_decl_set_hdf5_infer_size")


def op_decl_map_hdf5(frm, to, dim: int, file: str, name: str):
    return _declared(load().op_decl_map_hdf5(frm, to, int(dim), _b(file), _b(name)),
                     "op_decl_map_hdf5")


def op_decl_dat_hdf5(set_, dim: int, type_: str, file: str, name: str):
    return _declared(load().op_decl_dat_hdf5(set_, int(dim), _b(type_), _b(file), _b(name)),
                     "op_decl_dat_hdf5")


def op_get_const_hdf5(name: str, dim: int, type_: str, file: str) -> np.ndarray:
    out = np.zeros(dim, dtype=_H5_DTYPES[type_])
    _fails(lambda: load().op_get_const_hdf5(_b(name), int(dim), _b(type_), out.ctypes.data,
                                            _b(file)))
    return out


def op_dump_to_hdf5(file: str):
    _fails(lambda: load().op_dump_to_hdf5(_b(file)))


def op_write_const_hdf5(name: str, dim: int, type_: str, value, file: str):
    a = np.ascontiguousarray(value, dtype=_H5_DTYPES[type_]).reshape(-1)
    _fails(lambda: load().op_write_const_hdf5(_b(name), int(dim), _b(type_), a.ctypes.data,
                                              _b(file)))


def op_fetch_data_hdf5_file(dat, file: str, path: str | None = None):
    if path is None:
        _fails(lambda: load().op_fetch_data_hdf5_file(dat, _b(file)))
    else:
        _fails(lambda: load().op_fetch_data_hdf5_file_path(dat, _b(file), _b(path)))


def h5_info(file: str, path: str):
    """(shape, OP2 type name) of a dataset, or None when there is none."""
    rank = ctypes.c_int()
    dims = (ctypes.c_longlong * 8)()
    typ = ctypes.create_string_buffer(32)
    r = load().op2b_h5_info(_b(file), _b(path), ctypes.byref(rank), dims, typ, 32)
    if r < 0:
        _check(False, "op2b_h5_info")
    if r == 1:
        return None
    return tuple(dims[k] for k in range(rank.value)), typ.value.decode()


def h5_read(file: str, path: str, type_: str | None = None) -> np.ndarray:
    """A dataset's values as a numpy array of its shape (in `type_`, default
    the file's own type)."""
    info = h5_info(file, path)
    if info is None:
        raise Op2Error(f"no dataset {path} in {file}")
    shape, t = info
    t = type_ or t
    out = np.empty(shape, dtype=_H5_DTYPES[t])
    _check(load().op2b_h5_read(_b(file), _b(path), _b(t), out.ctypes.data, out.size) == 0,
           "op2b_h5_read")
    return out


def h5_write(file: str, path: str, data, type_: str | None = None):
    a = np.asarray(data, order="C")   # (ascontiguousarray would make a scalar 1-d)
    t = type_ or {np.dtype(np.int32): "int", np.dtype(np.int64): "long",
                  np.dtype(np.float32): "float", np.dtype(np.float64): "double"}[a.dtype]
    a = np.asarray(a, dtype=_H5_DTYPES[t], order="C")
    dims = (ctypes.c_longlong * max(a.ndim, 1))(*a.shape)
    _check(load().op2b_h5_write(_b(file), _b(path), _b(t), a.ndim, dims, a.ctypes.data) == 0,
           "op2b_h5_write")


def h5_set_attr(file: str, path: str, name: str, value, type_: str = "int"):
    if type_ == "string":
        b = value.encode()
        r = load().op2b_h5_set_attr(_b(file), _b(path), _b(name), b"string", len(b),
                                    ctypes.c_char_p(b))
    else:
        a = np.ascontiguousarray(value, dtype=_H5_DTYPES[type_]).reshape(-1)
        r = load().op2b_h5_set_attr(_b(file), _b(path), _b(name), _b(type_), a.size,
                                    a.ctypes.data)
    _check(r == 0, "op2b_h5_set_attr")


def h5_get_attr(file: str, path: str, name: str) -> str | None:
    buf = ctypes.create_string_buffer(4096)
    r = load().op2b_h5_get_attr(_b(file), _b(path), _b(name), buf, 4096)
    if r < 0:
        _check(False, "op2b_h5_get_attr")
    return None if r == 1 else buf.value.decode()


def h5_list(file: str) -> list[str]:
    n = load().op2b_h5_list(_b(file), None, 0)
    if n < 0:
        _check(False, "op2b_h5_list")
    buf = ctypes.create_string_buffer(int(n))
    load().op2b_h5_list(_b(file), buf, n)
    return [ln for ln in buf.value.decode().split("\n") if ln]


def op_get_size(set_) -> int:
    return load().op_get_size(set_)


def register_kernel(name: str, source: str | None):
    """Kernel source for a loop without a hand-written device kernel (compiled
    at its first op_par_loop call, op2b_register_kernel); None forgets it."""
    if load().op2b_register_kernel(_b(name), None if source is None else source.encode()) != 0:
        _check(False, "op2b_register_kernel")


def register_prelude(source: str):
    if load().op2b_register_prelude(source.encode()) != 0:
        _check(False, "op2b_register_prelude")


def set_option(key: str, value: int):
    if load().op2b_set_option(_b(key), int(value)) != 0:
        _check(False, "op2b_set_option")


def get_option(key: str) -> int:
    return load().op2b_get_option(_b(key))


def loop_stats(name: str):
    t, c, b, last = ctypes.c_double(), ctypes.c_long(), ctypes.c_double(), ctypes.c_double()
    if load().op2b_loop_stats(_b(name), ctypes.byref(t), ctypes.byref(c), ctypes.byref(b),
                              ctypes.byref(last)) != 0:
        return None
    return dict(total_ms=t.value, calls=c.value, bytes_per_call=b.value, last_ms=last.value)


def synchronize():
    rc = load().op2b_synchronize()
    if rc != 0:
        _check(False, "op2b_synchronize")
