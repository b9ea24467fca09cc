"""ctypes binding of the C ABI in include/vlx_b200.h (libvlx_b200.so).

The library is built in-tree (python -m veloxchem_b200.build).  There is no
fallback: if the library is missing or fails to load, every entry point raises.
"""

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / 'lib' / 'libvlx_b200.so'

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); every symbol declared in include/vlx_b200.h
SIGNATURES = {
    'vlx_b200_version': (ctypes.c_char_p, []),
    'vlx_b200_last_error': (ctypes.c_char_p, []),
    'vlx_b200_device_count': (ctypes.c_int, [_ip]),
    'vlx_b200_normalize_shell': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dp, _dp]),
    'vlx_b200_screener_create': (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                                _ip, _ip, _ip, _dp, _dp]),
    'vlx_b200_screener_destroy': (ctypes.c_int, [_vp]),
    'vlx_b200_screener_nao': (ctypes.c_int, [_vp, _ip]),
    'vlx_b200_screener_npairs': (ctypes.c_int, [_vp, _ip]),
    'vlx_b200_screener_pair_info': (ctypes.c_int, [_vp, _ip, _dp]),
    'vlx_b200_set_block_size_factor': (ctypes.c_int, [_vp, ctypes.c_int]),
    'vlx_b200_fock_build': (ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.c_char_p, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, _dp, _vp]),
    'vlx_b200_fock_build_local': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                                 ctypes.c_char_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                 _dp, _vp]),
    'vlx_b200_fock_build_multi': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.POINTER(_dp), ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_char_p), ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_int, ctypes.POINTER(_dp), _vp]),
    'vlx_b200_fock_build_device': (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_int, _vp, _vp]),
    'vlx_b200_fock_build_local_device': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                        ctypes.c_char_p, ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_int, _vp, _vp]),
    'vlx_b200_set_partition': (ctypes.c_int, [_vp, ctypes.c_int]),
    'vlx_b200_compute_eri': (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    'vlx_b200_boys_device': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]),
    'vlx_b200_fock_profile': (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_double, ctypes.c_int,
                                             _vp, _vp, ctypes.c_int, _vp, _ip]),
    'vlx_b200_fp64_peak': (ctypes.c_int, [ctypes.c_int, _dp]),
    'vlx_b200_one_electron': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_int,
                                             _ip, _ip, _ip, _dp, _dp, ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp]),
    'vlx_b200_one_electron_device': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_int,
                                             _ip, _ip, _ip, _dp, _dp, ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _vp, _vp]),
    'vlx_b200_set_fp32_threshold': (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    'vlx_b200_set_density_screening': (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    'vlx_b200_set_fp32_digestion': (ctypes.c_int, [_vp, ctypes.c_int]),
    'vlx_b200_fock_build_noalloc': (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_int, _vp, _vp]),
    'vlx_b200_mlp_linear': (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _vp]),
    'vlx_b200_mlp_linear_bf16': (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, _vp]),
    'vlx_b200_mlp_linear_backward': (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int,
                                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    'vlx_b200_mlp_mse': (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_longlong, ctypes.c_double, _vp]),
    'vlx_b200_adam_step': (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_longlong, ctypes.c_float, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_float, ctypes.c_int, _vp]),
    'vlx_b200_to_bf16': (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _vp]),
    'vlx_b200_set_work_threshold': (ctypes.c_int, [_vp, ctypes.c_int]),
    'vlx_b200_autotune': (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _ip]),
    'vlx_b200_batch_create': (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.c_int]),
    'vlx_b200_batch_destroy': (ctypes.c_int, [_vp]),
    'vlx_b200_batch_offsets': (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    'vlx_b200_batch_fock_build': (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp]),
}


class ClassProfile(ctypes.Structure):
    _fields_ = [('la', ctypes.c_int), ('lb', ctypes.c_int), ('lc', ctypes.c_int), ('ld', ctypes.c_int),
                ('table_driven', ctypes.c_int), ('device_ms', ctypes.c_double),
                ('shell_quartets', ctypes.c_longlong), ('prim_quartets', ctypes.c_longlong),
                ('flops', ctypes.c_double), ('fp32_quartets', ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneResult(ctypes.Structure):
    _fields_ = [('la', ctypes.c_int), ('lb', ctypes.c_int), ('lc', ctypes.c_int), ('ld', ctypes.c_int),
                ('table_driven', ctypes.c_int), ('segment', ctypes.c_int), ('best_ms', ctypes.c_double),
                ('default_ms', ctypes.c_double), ('blocks_per_sm', ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def autotune(screener, d_density_ptr, ithreshold=12, stream_ptr=None, max_classes=256):
    """Per-class work-item lengths for the screener's later builds; returns the choices."""
    arr = (TuneResult * max_classes)()
    n = ctypes.c_int(0)
    check(lib().vlx_b200_autotune(screener.handle, ctypes.c_void_p(d_density_ptr), int(ithreshold),
                                  ctypes.c_void_p(stream_ptr) if stream_ptr else None, max_classes,
                                  ctypes.cast(arr, ctypes.c_void_p), ctypes.byref(n)), 'autotune')
    return [arr[i].as_dict() for i in range(n.value)]


def fp64_peak(device=0):
    v = ctypes.c_double(0.0)
    check(lib().vlx_b200_fp64_peak(int(device), ctypes.byref(v)), 'fp64_peak')
    return v.value


def fock_profile(screener, d_density_ptr, d_fock_ptr, label='2jk', xfac=1.0, ithreshold=12, symmetric=True,
                 stream_ptr=None, max_classes=256):
    arr = (ClassProfile * max_classes)()
    n = ctypes.c_int(0)
    check(lib().vlx_b200_fock_profile(screener.handle, ctypes.c_void_p(d_density_ptr), int(symmetric),
                                      label.encode(), float(xfac), int(ithreshold), ctypes.c_void_p(d_fock_ptr),
                                      ctypes.c_void_p(stream_ptr) if stream_ptr else None, max_classes,
                                      ctypes.cast(arr, ctypes.c_void_p), ctypes.byref(n)), 'fock_profile')
    return [arr[i].as_dict() for i in range(n.value)]


class Stats(ctypes.Structure):
    _fields_ = [('device_ms', ctypes.c_double), ('total_ms', ctypes.c_double), ('shell_quartets', ctypes.c_longlong),
                ('prim_quartets', ctypes.c_longlong), ('kernel_launches', ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class NativeError(RuntimeError):
    pass


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NativeError('native library not built: %s (run python -m veloxchem_b200.build)' % LIB_PATH)
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(rc, what):
    if rc != 0:
        msg = lib().vlx_b200_last_error().decode(errors='replace')
        raise NativeError('%s failed (code %d): %s' % (what, rc, msg))


def dptr(a):
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def device_count():
    n = ctypes.c_int(0)
    rc = lib().vlx_b200_device_count(ctypes.byref(n))
    return n.value if rc == 0 else 0


def normalize_shell(l, exps, coefs):
    e = f64(exps)
    c = f64(coefs).copy()
    check(lib().vlx_b200_normalize_shell(int(l), len(e), dptr(e), dptr(c)), 'normalize_shell')
    return c


def one_electron(which, molecule, bra_basis, ket_basis=None, device=0):
    """S (which=0), T (1) or V (2) between bra_basis and ket_basis (default: bra)."""
    ket_basis = bra_basis if ket_basis is None else ket_basis
    z = i32(molecule.get_element_ids())
    xyz = f64(molecule.get_coordinates_in_bohr())
    ba, bl, bn, be, bc = [a if a.dtype == np.float64 else i32(a) for a in bra_basis.shell_table()]
    ka, kl, kn, ke, kc = [a if a.dtype == np.float64 else i32(a) for a in ket_basis.shell_table()]
    out = np.zeros((bra_basis.get_dimensions_of_basis(), ket_basis.get_dimensions_of_basis()))
    check(lib().vlx_b200_one_electron(int(device), int(which), len(z), iptr(z), dptr(xyz), len(ba), iptr(ba),
                                      iptr(bl), iptr(bn), dptr(f64(be)), dptr(f64(bc)), len(ka), iptr(ka), iptr(kl),
                                      iptr(kn), dptr(f64(ke)), dptr(f64(kc)), dptr(out)), 'one_electron')
    return out


def one_electron_device(which, molecule, bra_basis, out, device=0, stream=None):
    """S, T or V of bra_basis into the device tensor ``out`` (float64,
    nao x nao, contiguous) on torch's current stream (or ``stream``)."""
    import torch
    z = i32(molecule.get_element_ids())
    xyz = f64(molecule.get_coordinates_in_bohr())
    ba, bl, bn, be, bc = [a if a.dtype == np.float64 else i32(a) for a in bra_basis.shell_table()]
    if stream is None:
        stream = torch.cuda.current_stream(out.device).cuda_stream or 1
    check(lib().vlx_b200_one_electron_device(int(device), int(which), len(z), iptr(z), dptr(xyz), len(ba),
                                             iptr(ba), iptr(bl), iptr(bn), dptr(f64(be)), dptr(f64(bc)), len(ba),
                                             iptr(ba), iptr(bl), iptr(bn), dptr(f64(be)), dptr(f64(bc)),
                                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream)),
          'one_electron_device')
    return out


def boys_device(m, t, device=0):
    t = f64(t)
    out = np.zeros_like(t)
    check(lib().vlx_b200_boys_device(int(device), int(m), len(t), dptr(t), dptr(out)), 'boys_device')
    return out
