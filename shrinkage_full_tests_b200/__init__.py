"""B200-native resist-shrinkage operator — Python host mirror of the C ABI.

The operator (pky8903/shrinkage_full_tests)

    h = c * ( conv(Gx, g) * df/dx + conv(Gy, g) * df/dy ),   W = N - 2*erosion

and its derivatives run in hand-written sm_100a kernels inside
libsrk_b200.so (built in-tree by ``build.py``).  This module loads that
library through ctypes and exposes the reference's entry points under their
reference names with the reference's argument order; the workspace argument
``ws`` is an :class:`SrkPlan`.  Device buffers are torch tensors (or raw
device addresses given as ``int``); nothing here computes on the host, and
every entry point raises :class:`SrkError` if the library is missing or a
call fails.
"""
import ctypes
import os

__all__ = [
    "SrkError", "SrkPlan", "lib", "srkTrainingForward", "srkForwardOaS", "adjointSRK",
    "shrinkageTangentOaS", "shrinkageTangentAdjointOaS", "srkPrecomputeKernelFreq", "green_tensor",
    "forward", "vjp", "jvp", "SRK_ADJ_REFERENCE", "SRK_ADJ_TRUE",
]

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SRK_B200_LIB") or os.path.join(_PKG, "libsrk_b200.so")

SRK_OK, SRK_ERR_INVALID_ARG, SRK_ERR_UNSUPPORTED, SRK_ERR_ALLOC, SRK_ERR_TIMEOUT, SRK_ERR_CUDA = range(6)
SRK_F32, SRK_F16, SRK_BF16 = 0, 1, 2
SRK_ADJ_REFERENCE, SRK_ADJ_TRUE = 0, 1
SRK_SCHEDULE_PERSISTENT, SRK_SCHEDULE_THREE_PASS, SRK_SCHEDULE_DIRECT, SRK_SCHEDULE_TENSOR_ROWS = 0, 1, 2, 3


class SrkError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (_STATUS.get(status, status), message))
        self.status = status


_STATUS = {0: "SRK_OK", 1: "SRK_ERR_INVALID_ARG", 2: "SRK_ERR_UNSUPPORTED", 3: "SRK_ERR_ALLOC",
           4: "SRK_ERR_TIMEOUT", 5: "SRK_ERR_CUDA"}


class PlanInfo(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("W", ctypes.c_int), ("erosion", ctypes.c_int), ("B_max", ctypes.c_int),
                ("spectra_M", ctypes.c_int), ("dx", ctypes.c_float), ("tile_M", ctypes.c_int),
                ("tile_stride", ctypes.c_int), ("tiles", ctypes.c_int), ("tiles_adj", ctypes.c_int),
                ("chunk_wt", ctypes.c_int), ("scratch_bytes", ctypes.c_size_t), ("dtype", ctypes.c_int),
                ("schedule", ctypes.c_int), ("last_launches", ctypes.c_int), ("last_grid", ctypes.c_int),
                ("last_lag", ctypes.c_int), ("last_nslot", ctypes.c_int), ("last_spins", ctypes.c_ulonglong)]


_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double

# name -> argtypes (restype is srk_status = int unless listed in _RESTYPE)
_SIGS = {
    "srk_version": [],
    "srk_status_string": [_I],
    "srk_last_error": [],
    "srk_plan_create": [ctypes.POINTER(_P), _I, _I, _I, _F, _I, _I, _I, _I, ctypes.c_size_t],
    "srk_plan_destroy": [_P],
    "srk_plan_get_info": [_P, ctypes.POINTER(PlanInfo)],
    "srk_plan_set_adj_convention": [_P, _I],
    "srk_plan_set_schedule": [_P, _I],
    "srk_measure_cd": [_P, _I, _I, _I, _I, _P, _P, _P, _P],
    "srk_cd_after_shrinkage": [_P, _P, _I, _I, _I, _I, _F, _I, _I, _I, _P, _P, _P, _P],
    "srk_training_forward_noalloc": [_P, _P, _P, _P, _I, _I, _I, _F, _I, _P, _P],
    "srk_autotune": [_I, _I, _I, _F, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "srk_plan_set_persistent": [_P, _I, _I, _I],
    "srk_plan_sync": [_P, _P],
    "srk_debug_wait_selftest": [_P, ctypes.c_ulonglong, _P],
    "srk_plan_import_spectra": [_P, _P, _P, _P],
    "srk_plan_set_kernel": [_P, _P, _P, _I, _P],
    "srk_green_tensor": [_P, _P, _I, _D, _D, _D, _P],
    "srk_precompute_kernel_freq": [_P, _I, _I, _P, _P],
    "srk_training_forward": [_P, _P, _P, _P, _I, _I, _I, _F, _I, _P, _P, _P],
    "srk_training_forward_sync": [_P, _P, _P, _P, _I, _I, _I, _F, _I, _P, _P, _P],
    "srk_forward_oas": [_P, _P, _P, _P, _I, _I, _I, _F, _P, _P, _P, _P, _P],
    "srk_adjoint": [_P, _P, _P, _P, _P, _P, _I, _I, _I, _F, _P, _P, _P, _P],
    "srk_tangent": [_P, _P, _P, _P, _P, _P, _I, _I, _I, _F, _P, _P, _P],
    "srk_tangent_adjoint": [_P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _F, _P, _P, _P, _P],
    "srk_forward": [_P, _P, _I, _P, _P, _P],
    "srk_vjp": [_P, _P, _P, _I, _P, _P, _P, _P],
    "srk_jvp": [_P, _P, _P, _P, _I, _P, _P, _P],
    "srk_cd_strip": [_P, _P, _P, _P, _I, _I, _I, _I, _F, _I, _F, _I, _I, _I, _P, _P, _P, _P],
    "srk_grf": [_I, _I, _D, ctypes.c_ulonglong, _I, _P, _P],
    "srk_grf_filter": [_P, _I, _I, _D, _I, _P, _P],
    "srk_lns": [_I, _I, _P, _F, _F, _I, _P, _P],
    "srk_forward_oas_ragged": [_P, _P, _P, _P, _I, _P, _I, _F, _P, _P, _P],
    "srk_adjoint_ragged": [_P, _P, _P, _P, _P, _P, _I, _P, _I, _F, _P, _P, _P, _P],
    "srk_tangent_ragged": [_P, _P, _P, _P, _P, _P, _I, _P, _I, _F, _P, _P, _P],
    "srk_tangent_adjoint_ragged": [_P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _I, _F, _P, _P, _P, _P],
    "srk_forward_oas_slab": [_P, _P, _P, _P, _I, _I, _F, _I, _I, _P, _P, _P],
    "srk_tangent_slab": [_P, _P, _P, _P, _P, _P, _I, _I, _F, _I, _I, _P, _P, _P],
    "srk_adjoint_slab": [_P, _P, _P, _P, _P, _P, _I, _I, _F, _I, _I, _P, _P, _P, _P],
    "srk_tangent_adjoint_slab": [_P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _F, _I, _I, _P, _P, _P, _P],
}
# storage-typed forms (void* buffers in the plan's dtype): same argument types
for _n in ("srk_training_forward", "srk_forward_oas", "srk_adjoint", "srk_tangent", "srk_tangent_adjoint",
           "srk_forward", "srk_vjp", "srk_jvp"):
    _SIGS[_n + "_t"] = _SIGS[_n]
_RESTYPE = {"srk_version": _I, "srk_status_string": ctypes.c_char_p, "srk_last_error": ctypes.c_char_p}


def lib():
    """Load libsrk_b200.so (fails loudly if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SrkError(SRK_ERR_UNSUPPORTED, "libsrk_b200.so not built at %s (run __graft_entry__.build())"
                           % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, _I)
        _lib = L
    return _lib


def _check(status):
    if status != SRK_OK:
        raise SrkError(status, lib().srk_last_error().decode())


def _ptr(t):
    """Device address of a torch tensor (or pass-through int / None)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise SrkError(SRK_ERR_INVALID_ARG, "expected a CUDA tensor")
    if not t.is_contiguous():
        raise SrkError(SRK_ERR_INVALID_ARG, "expected a contiguous tensor")
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class SrkPlan:
    """Owns the scratch and spectra of one (N, W, erosion, dx) configuration;
    stands in for the reference's Srk*Workspace structs."""

    def __init__(self, N, W, erosion, dx=1.0, B_max=1, spectra_M=None, dtype=SRK_F32, tile_M=0,
                 scratch_budget=0):
        h = _P()
        _check(lib().srk_plan_create(ctypes.byref(h), N, W, erosion, dx, B_max,
                                     spectra_M if spectra_M is not None else N, dtype, tile_M, scratch_budget))
        self.handle = h.value
        self.N, self.W, self.erosion, self.dx, self.B_max = N, W, erosion, dx, B_max
        self.dtype = dtype

    def info(self):
        i = PlanInfo()
        _check(lib().srk_plan_get_info(self.handle, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in PlanInfo._fields_}

    def set_adj_convention(self, conv):
        _check(lib().srk_plan_set_adj_convention(self.handle, conv))

    def set_schedule(self, schedule):
        _check(lib().srk_plan_set_schedule(self.handle, schedule))

    def set_persistent(self, lag=0, grid=0, prefetch=1):
        _check(lib().srk_plan_set_persistent(self.handle, lag, grid, prefetch))

    def sync(self, stream=None):
        """Synchronise and raise SrkError(SRK_ERR_TIMEOUT) if a bounded
        device-side wait of the last launch gave up."""
        _check(lib().srk_plan_sync(self.handle, _stream(stream)))

    def wait_selftest(self, spin_limit=1 << 12, stream=None):
        """Return the status of the bounded-wait self test (SRK_ERR_TIMEOUT expected)."""
        return lib().srk_debug_wait_selftest(self.handle, spin_limit, _stream(stream))

    def import_spectra(self, Gx_freq, Gy_freq, stream=None):
        _check(lib().srk_plan_import_spectra(self.handle, _ptr(Gx_freq), _ptr(Gy_freq), _stream(stream)))

    def set_kernel(self, Kx, Ky, stream=None):
        _check(lib().srk_plan_set_kernel(self.handle, _ptr(Kx), _ptr(Ky), Kx.shape[-1], _stream(stream)))

    def destroy(self):
        if self.handle:
            lib().srk_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


SRK_TILE_AUTOTUNE = -1


def autotune(N, W, erosion, dx=1.0, B=1, dtype=SRK_F32):
    """(tile_M, schedule) the library picks for this configuration (timed once
    per device, then cached on disk)."""
    m, sc = _I(), _I()
    _check(lib().srk_autotune(N, W, erosion, dx, B, dtype, ctypes.byref(m), ctypes.byref(sc)))
    return m.value, sc.value


def _entry(name, ws):
    """fp32 plans use the reference-typed (float*) entry point, fp16/bf16
    plans the storage-typed _t form."""
    return getattr(lib(), name if ws.dtype == SRK_F32 else name + "_t")


def srkTrainingForward(E, I, Gx_freq, Gy_freq, N, W, erosion, dx, B, stream, R, ws):
    _check(_entry("srk_training_forward", ws)(_ptr(E), _ptr(I), _ptr(Gx_freq), _ptr(Gy_freq), N, W, erosion, dx, B,
                                              _stream(stream), _ptr(R), ws.handle))


def srkForwardOaS(E, I, Gx_freq, Gy_freq, N, W, erosion, dx, stream, R, ws, ux=None, uy=None):
    _check(_entry("srk_forward_oas", ws)(_ptr(E), _ptr(I), _ptr(Gx_freq), _ptr(Gy_freq), N, W, erosion, dx,
                                         _stream(stream), _ptr(R), ws.handle, _ptr(ux), _ptr(uy)))


def adjointSRK(v, ux, uy, I, Gx_freq, Gy_freq, N, W, erosion, dx, stream, dLdI, dLdE, ws):
    _check(_entry("srk_adjoint", ws)(_ptr(v), _ptr(ux), _ptr(uy), _ptr(I), _ptr(Gx_freq), _ptr(Gy_freq), N, W,
                                     erosion, dx, _stream(stream), _ptr(dLdI), _ptr(dLdE), ws.handle))


def shrinkageTangentOaS(f, g, df, dg, Gx_freq, Gy_freq, N, W, erosion, dx, stream, dh, ws):
    _check(_entry("srk_tangent", ws)(_ptr(f), _ptr(g), _ptr(df), _ptr(dg), _ptr(Gx_freq), _ptr(Gy_freq), N, W,
                                     erosion, dx, _stream(stream), _ptr(dh), ws.handle))


def shrinkageTangentAdjointOaS(f, g, df, dg, lam_h, dlam_h, Gx_freq, Gy_freq, N, W, erosion, dx, stream,
                               dLam_f, dLam_g, ws):
    _check(_entry("srk_tangent_adjoint", ws)(_ptr(f), _ptr(g), _ptr(df), _ptr(dg), _ptr(lam_h), _ptr(dlam_h),
                                             _ptr(Gx_freq), _ptr(Gy_freq), N, W, erosion, dx, _stream(stream),
                                             _ptr(dLam_f), _ptr(dLam_g), ws.handle))


def _sizes(Ns):
    Ns = [int(n) for n in Ns]
    return len(Ns), (ctypes.c_int * max(1, len(Ns)))(*Ns)


# ---- ragged batches: images of different N concatenated in every buffer
# (Ns[b]^2 elements per image in N-sized buffers, (Ns[b]-2e)^2 in W-sized ones)
def srkForwardOaSRagged(E, I, Gx_freq, Gy_freq, Ns, erosion, dx, stream, R, ws):
    B, arr = _sizes(Ns)
    _check(lib().srk_forward_oas_ragged(_ptr(E), _ptr(I), _ptr(Gx_freq), _ptr(Gy_freq), B, arr, erosion, dx,
                                        _stream(stream), _ptr(R), ws.handle))


def adjointSRKRagged(v, ux, uy, I, Gx_freq, Gy_freq, Ns, erosion, dx, stream, dLdI, dLdE, ws):
    B, arr = _sizes(Ns)
    _check(lib().srk_adjoint_ragged(_ptr(v), _ptr(ux), _ptr(uy), _ptr(I), _ptr(Gx_freq), _ptr(Gy_freq), B, arr,
                                    erosion, dx, _stream(stream), _ptr(dLdI), _ptr(dLdE), ws.handle))


def shrinkageTangentOaSRagged(f, g, df, dg, Gx_freq, Gy_freq, Ns, erosion, dx, stream, dh, ws):
    B, arr = _sizes(Ns)
    _check(lib().srk_tangent_ragged(_ptr(f), _ptr(g), _ptr(df), _ptr(dg), _ptr(Gx_freq), _ptr(Gy_freq), B, arr,
                                    erosion, dx, _stream(stream), _ptr(dh), ws.handle))


def shrinkageTangentAdjointOaSRagged(f, g, df, dg, lam_h, dlam_h, Gx_freq, Gy_freq, Ns, erosion, dx, stream,
                                     dLam_f, dLam_g, ws):
    B, arr = _sizes(Ns)
    _check(lib().srk_tangent_adjoint_ragged(_ptr(f), _ptr(g), _ptr(df), _ptr(dg), _ptr(lam_h), _ptr(dlam_h),
                                            _ptr(Gx_freq), _ptr(Gy_freq), B, arr, erosion, dx, _stream(stream),
                                            _ptr(dLam_f), _ptr(dLam_g), ws.handle))


# ---- column slabs of one image: every tensor's data pointer addresses column
# c0 of its array (a view such as buf[k:] of a halo'd column buffer), with the
# halo columns of the C declarations readable around it
def srkForwardOaSSlab(E, I, Gx_freq, Gy_freq, N, erosion, dx, c0, c1, stream, R, ws):
    _check(lib().srk_forward_oas_slab(_ptr(E), _ptr(I), _ptr(Gx_freq), _ptr(Gy_freq), N, erosion, dx, c0, c1,
                                      _stream(stream), _ptr(R), ws.handle))


def shrinkageTangentOaSSlab(f, g, df, dg, Gx_freq, Gy_freq, N, erosion, dx, c0, c1, stream, dh, ws):
    _check(lib().srk_tangent_slab(_ptr(f), _ptr(g), _ptr(df), _ptr(dg), _ptr(Gx_freq), _ptr(Gy_freq), N, erosion,
                                  dx, c0, c1, _stream(stream), _ptr(dh), ws.handle))


def adjointSRKSlab(v, ux, uy, I, Gx_freq, Gy_freq, N, erosion, dx, c0, c1, stream, dLdI, dLdE, ws):
    _check(lib().srk_adjoint_slab(_ptr(v), _ptr(ux), _ptr(uy), _ptr(I), _ptr(Gx_freq), _ptr(Gy_freq), N, erosion,
                                  dx, c0, c1, _stream(stream), _ptr(dLdI), _ptr(dLdE), ws.handle))


def shrinkageTangentAdjointOaSSlab(f, g, df, dg, lam_h, dlam_h, Gx_freq, Gy_freq, N, erosion, dx, c0, c1, stream,
                                   dLam_f, dLam_g, ws):
    _check(lib().srk_tangent_adjoint_slab(_ptr(f), _ptr(g), _ptr(df), _ptr(dg), _ptr(lam_h), _ptr(dlam_h),
                                          _ptr(Gx_freq), _ptr(Gy_freq), N, erosion, dx, c0, c1, _stream(stream),
                                          _ptr(dLam_f), _ptr(dLam_g), ws.handle))


# ---- synthetic inputs on the device
def grf(out, ell, seed, minmax=True, stream=None):
    """Gaussian random fields into out [B][N][N] (float32, CUDA): image b is
    keyed by seed + b."""
    B, N = (1, out.shape[-1]) if out.dim() == 2 else (out.shape[0], out.shape[-1])
    _check(lib().srk_grf(B, N, float(ell), int(seed), 1 if minmax else 0, _stream(stream), _ptr(out)))


def grf_filter(noise, out, ell, minmax=False, stream=None):
    """Filter caller noise [B][Np][Np] into out [B][N][N]."""
    B, N = (1, out.shape[-1]) if out.dim() == 2 else (out.shape[0], out.shape[-1])
    _check(lib().srk_grf_filter(_ptr(noise), B, N, float(ell), 1 if minmax else 0, _stream(stream), _ptr(out)))


def lns(out, kinds, sigma_px, period_px=0.0, num_nbrs=4, stream=None):
    """Line/space patterns into out [B][N][N]; kinds[b] 0 = vertical, 1 = horizontal."""
    B, arr = _sizes(kinds)
    _check(lib().srk_lns(B, out.shape[-1], arr, float(sigma_px), float(period_px), num_nbrs, _stream(stream),
                         _ptr(out)))


def srkPrecomputeKernelFreq(K, kw, kh, M, G_freq, stream=None):
    """Spectrum of a (kw x kh, kw == kh) device kernel at size M, reference layout."""
    if kw != kh:
        raise SrkError(SRK_ERR_UNSUPPORTED, "square kernels only")
    _check(lib().srk_precompute_kernel_freq(_ptr(K), kw, M, _ptr(G_freq), _stream(stream)))


def green_tensor(Kx, Ky, gamma, R_w, dx, stream=None):
    """Fill device tensors Kx, Ky (KW x KW) with the FP64-evaluated Green's tensor."""
    _check(lib().srk_green_tensor(_ptr(Kx), _ptr(Ky), Kx.shape[-1], gamma, R_w, dx, _stream(stream)))


def forward(f, g, B, h, ws, stream=None):
    _check(_entry("srk_forward", ws)(_ptr(f), _ptr(g), B, _stream(stream), _ptr(h), ws.handle))


def vjp(v, f, g, B, dLdf, dLdg, ws, stream=None):
    _check(_entry("srk_vjp", ws)(_ptr(v), _ptr(f), _ptr(g), B, _stream(stream), _ptr(dLdf), _ptr(dLdg), ws.handle))


def jvp(f, g, df, dg, B, dh, ws, stream=None):
    _check(_entry("srk_jvp", ws)(_ptr(f), _ptr(g), _ptr(df), _ptr(dg), B, _stream(stream), _ptr(dh), ws.handle))


def measure_cd(sig, L=16, A=8, stream=None):
    """(left, right, cd) device tensors [B] for signals sig [B][n]
    (MeasureCD_Batched semantics, pixels)."""
    import torch
    B, n = sig.shape
    out = [torch.empty(B, device=sig.device, dtype=torch.float32) for _ in range(3)]
    _check(lib().srk_measure_cd(_ptr(sig), B, n, L, A, _stream(stream), *[_ptr(t) for t in out]))
    return tuple(out)


def cd_after_shrinkage(E, R, N, W, erosion, coeff, axis, L=16, A=8, stream=None):
    """CD of the centre row (axis 0) or column (axis 1) of E_crop + coeff*R."""
    import torch
    B = E.shape[0]
    out = [torch.empty(B, device=E.device, dtype=torch.float32) for _ in range(3)]
    _check(lib().srk_cd_after_shrinkage(_ptr(E), _ptr(R), B, N, W, erosion, coeff, axis, L, A, _stream(stream),
                                        *[_ptr(t) for t in out]))
    return tuple(out)


def cd_strip(E, I, Kx, Ky, N, W, erosion, dx, coeff, axis, L=16, A=8, stream=None):
    """CD of the centre row (axis 0) or column (axis 1) of E_crop + coeff*R,
    with R computed on that line only (spatial kernels Kx, Ky, KW x KW)."""
    import torch
    B = E.shape[0]
    out = [torch.empty(B, device=E.device, dtype=torch.float32) for _ in range(3)]
    _check(lib().srk_cd_strip(_ptr(E), _ptr(I), _ptr(Kx), _ptr(Ky), Kx.shape[-1], N, W, erosion, dx, B, coeff, axis,
                              L, A, _stream(stream), *[_ptr(t) for t in out]))
    return tuple(out)
