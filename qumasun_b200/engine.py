"""ctypes binding of the engine's C ABI (include/qumasun_b200.h).

Mirrors the reference's operator interface for the H|psi> path: a Hamiltonian
is built once per geometry from the reference's cube tables
(PseudoPotIntegrator::UpdatePosition, PseudoPotOperator.h:453-466) and then
applied to blocks of states (the OpeA callback of qumasun_single.lobpcg.h:19-23,
batched). There is no CPU path: if the shared library or a CUDA device is
missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqumasun_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_longlong)

QG_OK = 0
STATUS = {
    0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "device out of memory",
    -4: "Gram matrix not positive definite", -5: "bounded device wait timed out",
    -6: "non-finite value", -7: "unsupported shape or option", -8: "CUDA library error",
    -9: "not converged within the iteration limit",
}


class QGError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)} ({status}) {detail}".strip())


class HamiltonianDesc(C.Structure):
    """qg_hamiltonian_desc."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double),
        ("fd_order", C.c_int),
        ("V", _dp),
        ("n_atoms", C.c_int),
        ("atom_pos", _dp),
        ("n_proj", C.c_int),
        ("proj_l", _ip),
        ("proj_E", _dp),
        ("cube", _ip),
        ("w_data", _dp),
        ("w_off", _lp),
        ("n_lm", C.c_int),
        ("ylm_data", _dp),
        ("ylm_off", _lp),
        ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
    ]


class LobpcgOptions(C.Structure):
    """qg_lobpcg_options."""

    _fields_ = [("max_iter", C.c_int), ("tol", C.c_double), ("first_call", C.c_int),
                ("precision", C.c_int), ("verbose", C.c_int), ("precond", C.c_int),
                ("precond_shift", C.c_double), ("n_converge", C.c_int)]


class LobpcgReport(C.Structure):
    """qg_lobpcg_report."""

    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("max_residual", C.c_double),
                ("ms_total", C.c_double), ("ms_hamiltonian", C.c_double), ("ms_gram", C.c_double),
                ("ms_eigensolve", C.c_double), ("ms_rotate", C.c_double), ("ms_vector", C.c_double),
                ("restarts", C.c_int), ("mixed_iterations", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def lib():
    """The loaded engine library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m qumasun_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.qg_status_string.restype = C.c_char_p
        L.qg_last_error.restype = C.c_char_p
        L.qg_context_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.qg_context_destroy.argtypes = [vp]
        L.qg_context_set_stream.argtypes = [vp, vp]
        L.qg_context_synchronize.argtypes = [vp]
        L.qg_hamiltonian_create.argtypes = [vp, C.POINTER(HamiltonianDesc), C.POINTER(vp)]
        L.qg_hamiltonian_destroy.argtypes = [vp]
        L.qg_hamiltonian_set_kvector.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.qg_hamiltonian_apply_d.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong]
        L.qg_hamiltonian_apply_f.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong]
        L.qg_hamiltonian_apply_host_d.argtypes = [vp, C.c_int, vp, vp]
        L.qg_hamiltonian_apply_timed_d.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong,
                                                   C.POINTER(C.c_float)]
        L.qg_hamiltonian_apply_z.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong]
        L.qg_hamiltonian_apply_host_z.argtypes = [vp, C.c_int, vp, vp]
        L.qg_hamiltonian_apply_zk.argtypes = [vp, C.c_int, _dp, C.c_int, vp, C.c_longlong, C.c_longlong, vp,
                                              C.c_longlong, C.c_longlong]
        L.qg_hamiltonian_apply_zf.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong]
        L.qg_hamiltonian_apply_zkf.argtypes = [vp, C.c_int, _dp, C.c_int, vp, C.c_longlong, C.c_longlong, vp,
                                               C.c_longlong, C.c_longlong]
        L.qg_hamiltonian_apply_timed_z.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong,
                                                   C.POINTER(C.c_float)]
        L.qg_hamiltonian_launches_per_apply.argtypes = [vp, C.c_int]
        L.qg_hamiltonian_set_stencil_kernel.argtypes = [vp, C.c_int]
        L.qg_hamiltonian_set_nonlocal_blocking.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.qg_hamiltonian_set_gram_reuse.argtypes = [vp, C.c_int]
        L.qg_hamiltonian_test_stall.argtypes = [vp, C.c_int]
        L.qg_hamiltonian_autotune_d.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong, _ip,
                                                C.POINTER(C.c_float)]
        L.qg_hamiltonian_autotune_f.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong, _ip,
                                                C.POINTER(C.c_float)]
        L.qg_context_take_device_status.argtypes = [vp]
        L.qg_hamiltonian_apply_noalloc_d.argtypes = [vp, C.c_int, vp, C.c_longlong, vp, C.c_longlong]
        L.qg_noalloc_scratch_capacity.restype = C.c_size_t
        L.qg_sygv_small_batched_d.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_int, C.c_longlong, vp, vp, _ip]
        L.qg_hegv_small_batched_z.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_int, C.c_longlong, vp, vp, _ip]
        L.qg_gram_small_d.argtypes = [vp, C.c_longlong, C.c_int, C.c_int, vp, vp, C.c_double, vp]
        L.qg_lobpcg_d.argtypes = [vp, C.POINTER(LobpcgOptions), C.c_int, _dp, vp, vp, C.POINTER(LobpcgReport)]
        L.qg_gram_mixed_d.argtypes = [vp, C.c_longlong, C.c_int, vp, vp, C.c_double, vp, C.c_int]
        L.qg_learned_create.argtypes = [vp, C.POINTER(vp)]
        L.qg_learned_destroy.argtypes = [vp]
        L.qg_learned_set_params.argtypes = [vp, C.POINTER(C.c_float), C.c_int]
        L.qg_learned_get_params.argtypes = [vp, C.POINTER(C.c_float), C.c_int]
        L.qg_learned_apply_d.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_longlong, vp, C.c_double,
                                         vp, C.c_longlong, C.c_int]
        L.qg_learned_set_tensor_cores.argtypes = [vp, C.c_int]
        L.qg_learned_gradient.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_longlong, vp, C.c_double,
                                          vp, C.c_longlong, C.POINTER(C.c_double), C.POINTER(C.c_float)]
        L.qg_learned_train_step.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_longlong, vp,
                                            C.c_double, vp, C.c_longlong, C.c_float, C.POINTER(C.c_double)]
        L.qg_hamiltonian_set_learned.argtypes = [vp, vp, C.c_double]
        L.qg_hamiltonian_precondition_d.argtypes = [vp, C.c_int, vp, C.c_longlong, C.c_double]
        L.qg_lobpcg_z.argtypes = [vp, C.POINTER(LobpcgOptions), C.c_int, _dp, vp, vp, C.POINTER(LobpcgReport)]
        L.qg_lobpcg_zk_device.argtypes = [vp, C.POINTER(LobpcgOptions), C.c_int, _dp, C.c_int, _dp, vp, vp,
                                          C.POINTER(LobpcgReport)]
        L.qg_lobpcg_z_device.argtypes = [vp, C.POINTER(LobpcgOptions), C.c_int, _dp, vp, vp,
                                         C.POINTER(LobpcgReport)]
        L.qg_lobpcg_d_device.argtypes = [vp, C.POINTER(LobpcgOptions), C.c_int, _dp, vp, vp,
                                         C.POINTER(LobpcgReport)]
        L.qg_lobpcg_cells_device.argtypes = [C.c_int, C.POINTER(vp), C.POINTER(LobpcgOptions), _ip,
                                             C.POINTER(_dp), C.POINTER(vp), C.POINTER(vp),
                                             C.POINTER(LobpcgReport), _ip]
        L.qg_density_d.argtypes = [vp, C.c_longlong, C.c_int, vp, C.c_longlong, _dp, vp, C.c_int]
        L.qg_density_z.argtypes = [vp, C.c_longlong, C.c_int, vp, C.c_longlong, _dp, vp, C.c_int]
        L.qg_occupancy.argtypes = [C.c_double, C.c_int, _dp, C.c_int, _dp, _dp]
        L.qg_occupancy_spin.argtypes = [C.c_double, C.c_int, _dp, _dp, C.c_int, _dp, _dp, _dp]
        L.qg_poisson_create.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.POINTER(vp)]
        L.qg_poisson_destroy.argtypes = [vp]
        L.qg_potential_lda_d.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        L.qg_td_taylor4_z.argtypes = [vp, C.c_int, C.c_double, vp, C.c_longlong]
        L.qg_nonlocal_force_d.argtypes = [vp, C.c_int, vp, C.c_longlong, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def check(status, where):
    if status != QG_OK:
        detail = lib().qg_last_error().decode(errors="replace")
        raise QGError(status, where, detail)


class Context:
    """A device context (qg_context): one CUDA device, one stream."""

    def __init__(self, device=0):
        self.h = C.c_void_p()
        check(lib().qg_context_create(device, C.byref(self.h)), "qg_context_create")
        self.device = device
        self.children = weakref.WeakSet()

    def set_stream(self, stream_ptr):
        check(lib().qg_context_set_stream(self.h, C.c_void_p(stream_ptr)), "qg_context_set_stream")

    def synchronize(self):
        check(lib().qg_context_synchronize(self.h), "qg_context_synchronize")

    def take_device_status(self):
        return lib().qg_context_take_device_status(self.h)

    def use_torch_stream(self):
        """Issue the engine's work on torch's current CUDA stream (orders it
        with the surrounding torch operations)."""
        import torch
        self.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def close(self):
        if self.h:
            for child in list(self.children):
                child.close()
            lib().qg_context_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _dev(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def density(ctx, X, occ, rho=None, accumulate=False, complex_states=False):
    """rho (+)= sum_s occ[s] |psi_s|^2 on the device (qg_density_d / _z): X a CUDA float64
    tensor (ns, N) of real states or (ns, 2N) of {re, im} states, occ host values."""
    import torch
    occ = np.ascontiguousarray(occ, dtype=np.float64)
    ns = X.shape[0]
    N = X.shape[1] // (2 if complex_states else 1)
    if occ.shape[0] != ns:
        raise ValueError("one occupation per state")
    if not (X.is_cuda and X.dtype == torch.float64 and X.is_contiguous()):
        raise TypeError("X must be a contiguous float64 CUDA tensor")
    if rho is None:
        rho = torch.zeros(N, dtype=torch.float64, device=X.device)
        accumulate = False
    ctx.use_torch_stream()
    fn = lib().qg_density_z if complex_states else lib().qg_density_d
    check(fn(ctx.h, N, ns, _dev(X), X.shape[1], occ.ctypes.data_as(_dp), _dev(rho), 1 if accumulate else 0),
          "qg_density")
    return rho


def occupancy(kbT, ev, n_electrons, ev_down=None):
    """Fermi occupations by bisection on mu (qg_occupancy / qg_occupancy_spin).
    Returns (occ, mu) or ((occ_up, occ_down), mu) with ev_down."""
    ev = np.ascontiguousarray(ev, dtype=np.float64)
    mu = C.c_double()
    if ev_down is None:
        occ = np.zeros_like(ev)
        check(lib().qg_occupancy(kbT, len(ev), ev.ctypes.data_as(_dp), int(n_electrons), occ.ctypes.data_as(_dp),
                                 C.byref(mu)), "qg_occupancy")
        return occ, mu.value
    ed = np.ascontiguousarray(ev_down, dtype=np.float64)
    ou, od = np.zeros_like(ev), np.zeros_like(ed)
    check(lib().qg_occupancy_spin(kbT, len(ev), ev.ctypes.data_as(_dp), ed.ctypes.data_as(_dp), int(n_electrons),
                                  ou.ctypes.data_as(_dp), od.ctypes.data_as(_dp), C.byref(mu)), "qg_occupancy_spin")
    return (ou, od), mu.value


class Poisson:
    """FFT Poisson + LDA potential builder of one periodic grid (qg_poisson)."""

    def __init__(self, ctx: Context, grid, h):
        self.ctx = ctx
        self.N = int(grid[0] * grid[1] * grid[2])
        self.h = C.c_void_p()
        check(lib().qg_poisson_create(ctx.h, int(grid[0]), int(grid[1]), int(grid[2]), float(h[0]), float(h[1]),
                                      float(h[2]), C.byref(self.h)), "qg_poisson_create")
        self._fin = weakref.finalize(self, lib().qg_poisson_destroy, self.h)

    def potential(self, rho, vext, pcc=None, parts=False):
        """V_tot (and with parts=True also V_hart, V_x, V_c) from CUDA float64 tensors of N values."""
        import torch
        for t, n in ((rho, "rho"), (vext, "vext"), (pcc, "pcc")):
            if t is not None and not (t.is_cuda and t.dtype == torch.float64 and t.numel() == self.N
                                      and t.is_contiguous()):
                raise TypeError(f"{n} must be a contiguous float64 CUDA tensor of {self.N} values")
        out = [torch.empty_like(rho) for _ in range(4 if parts else 1)]
        extra = [_dev(o) for o in out[1:]] + [None] * (3 - len(out[1:]))
        self.ctx.use_torch_stream()
        check(lib().qg_potential_lda_d(self.h, _dev(rho), _dev(pcc), _dev(vext), _dev(out[0]), *extra),
              "qg_potential_lda_d")
        return tuple(out) if parts else out[0]

    def close(self):
        self._fin()


def sygv_small_batched(ctx, A, B):
    """Batched A z = lambda B z for torch CUDA float64 tensors (batch, k, k) (symmetric;
    lower triangles read). Returns (w (batch, k), Z (batch, k, k) columns = eigenvectors, info)."""
    import torch
    bsz, k, _ = A.shape
    At = A.transpose(1, 2).contiguous()   # column-major per problem
    Bt = B.transpose(1, 2).contiguous()
    w = torch.empty(bsz, k, dtype=torch.float64, device=A.device)
    Z = torch.empty(bsz, k, k, dtype=torch.float64, device=A.device)
    info = np.zeros(bsz, dtype=np.int32)
    ctx.use_torch_stream()
    check(lib().qg_sygv_small_batched_d(ctx.h, bsz, k, C.c_void_p(At.data_ptr()), C.c_void_p(Bt.data_ptr()), k,
                                        k * k, C.c_void_p(w.data_ptr()), C.c_void_p(Z.data_ptr()),
                                        info.ctypes.data_as(_ip)), "qg_sygv_small_batched_d")
    return w, Z.transpose(1, 2), info


def lobpcg_cells(hams, Xs, Ps=None, max_iter=2000, tol=1.0e-10, first=True, precond=1, shift=1.0,
                 n_converge=None, precision=0):
    """Real LOBPCG on several independent cells at once (qg_lobpcg_cells_device).

    hams: Hamiltonians, each on its own Context; Xs: float64 CUDA tensors (ns_c, N_c),
    overwritten with the eigenvectors; Ps: matching tensors (or None on a first call);
    n_converge: per-cell counts of states that must converge (None: all). Each cell's
    context is put on its own CUDA stream so that the solves overlap on the GPU.
    Returns (list of dict(ev, report, status), overall status)."""
    import torch
    n = len(hams)
    assert n == len(Xs) and len({id(h.ctx) for h in hams}) == n, "one context per cell"
    for X in Xs:
        assert X.is_cuda and X.dtype == torch.float64 and X.is_contiguous()
    # the costliest cells (grid points x states, the top half) run on high-priority
    # streams: their solves are the critical path, the small cells fill the gaps
    cost = [X.shape[0] * X.shape[1] for X in Xs]
    cut = sorted(cost)[len(cost) // 2]
    streams = [torch.cuda.Stream(device=X.device, priority=-1 if c >= cut else 0) for X, c in zip(Xs, cost)]
    torch.cuda.synchronize()  # inputs written on other streams are complete
    for h, s in zip(hams, streams):
        h.ctx.set_stream(s.cuda_stream)
        h.ctx.cells_stream = s  # keeps the stream alive while the context may use it
    ncs = [0] * n if n_converge is None else list(n_converge)
    opts = (LobpcgOptions * n)(*[LobpcgOptions(max_iter, tol, 1 if first else 0, precision, 0, precond, shift,
                                               ncs[c]) for c in range(n)])
    reps = (LobpcgReport * n)()
    ns = np.array([X.shape[0] for X in Xs], dtype=np.int32)
    evs = [np.zeros(int(k)) for k in ns]
    ev_ptrs = (_dp * n)(*[e.ctypes.data_as(_dp) for e in evs])
    x_ptrs = (C.c_void_p * n)(*[X.data_ptr() for X in Xs])
    p_ptrs = (C.c_void_p * n)(*[(P.data_ptr() if P is not None else 0) for P in (Ps or [None] * n)])
    h_ptrs = (C.c_void_p * n)(*[h.h.value if isinstance(h.h, C.c_void_p) else h.h for h in hams])
    status = np.zeros(n, dtype=np.int32)
    rc = lib().qg_lobpcg_cells_device(n, h_ptrs, opts, ns.ctypes.data_as(_ip), ev_ptrs, x_ptrs, p_ptrs, reps,
                                      status.ctypes.data_as(_ip))
    for st in status:
        if st not in (QG_OK, -9):
            check(int(st), "qg_lobpcg_cells_device")
    out = [dict(ev=evs[c], report=reps[c].as_dict(), status=int(status[c])) for c in range(n)]
    return out, rc


def hegv_small_batched(ctx, A, B):
    """Batched Hermitian A z = lambda B z for torch CUDA complex128 tensors (batch, k, k)
    (lower triangles read). Returns (w (batch, k), Z (batch, k, k) columns = eigenvectors, info)."""
    import torch
    bsz, k, _ = A.shape
    At = A.transpose(1, 2).contiguous()   # column-major per problem
    Bt = B.transpose(1, 2).contiguous()
    w = torch.empty(bsz, k, dtype=torch.float64, device=A.device)
    Z = torch.empty(bsz, k, k, dtype=torch.complex128, device=A.device)
    info = np.zeros(bsz, dtype=np.int32)
    ctx.use_torch_stream()
    check(lib().qg_hegv_small_batched_z(ctx.h, bsz, k, C.c_void_p(At.data_ptr()), C.c_void_p(Bt.data_ptr()), k,
                                        k * k, C.c_void_p(w.data_ptr()), C.c_void_p(Z.data_ptr()),
                                        info.ctypes.data_as(_ip)), "qg_hegv_small_batched_z")
    return w, Z.transpose(1, 2), info


class LearnedPreconditioner:
    """The learned LOBPCG preconditioner network (qg_learned_*): 4 periodic 3^3
    convolutions 2 -> 16 -> 16 -> 16 -> 1 on [r / rms(r), V / vscale]; LOBPCG with
    precond=2 uses w = T r + rms(r) * net(...). Parameters start at zero."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.h = C.c_void_p()
        check(lib().qg_learned_create(ctx.h, C.byref(self.h)), "qg_learned_create")
        self.n_params = lib().qg_learned_num_params()
        ctx.children.add(self)

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        check(lib().qg_learned_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size),
              "qg_learned_set_params")

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        check(lib().qg_learned_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size),
              "qg_learned_get_params")
        return p

    @staticmethod
    def _check(grid, R, V, **blocks):
        """The network reads R (ns, nx*ny*nz) and V (nx*ny*nz) and reads or writes the
        other blocks whole: contiguous float64 CUDA tensors on one device, or a TypeError
        / ValueError before the library is called."""
        import torch
        N = int(grid[0]) * int(grid[1]) * int(grid[2])
        for name, T in (("R", R), ("V", V), *blocks.items()):
            if not isinstance(T, torch.Tensor) or not T.is_cuda or T.dtype != torch.float64:
                raise TypeError(f"{name} must be a float64 CUDA tensor")
            if not T.is_contiguous():
                raise ValueError(f"{name} must be contiguous")
            if T.device != R.device:
                raise ValueError(f"{name} is on {T.device}, R on {R.device}")
        if R.dim() != 2 or R.shape[1] != N:
            raise ValueError(f"R has shape {tuple(R.shape)}, expected (ns, {N})")
        if V.numel() != N:
            raise ValueError(f"V has {V.numel()} elements, expected {N}")
        for name, T in blocks.items():
            if T.shape != R.shape:
                raise ValueError(f"{name} has shape {tuple(T.shape)}, R {tuple(R.shape)}")

    def set_tensor_cores(self, on: bool):
        """Run the forward layers on the tensor cores (the default, where nx is a
        multiple of 8) or on the CUDA-core kernels."""
        check(lib().qg_learned_set_tensor_cores(self.h, 1 if on else 0), "qg_learned_set_tensor_cores")

    def apply(self, grid, R, V, vscale, out=None, accumulate=False):
        """out (+)= NN(R) for float64 CUDA tensors R (ns, N), V (N,)."""
        import torch
        if out is None:
            out = torch.zeros_like(R)
        self._check(grid, R, V, out=out)
        self.ctx.use_torch_stream()
        check(lib().qg_learned_apply_d(self.h, grid[0], grid[1], grid[2], R.shape[0], C.c_void_p(R.data_ptr()),
                                       R.shape[1], C.c_void_p(V.data_ptr()), float(vscale), C.c_void_p(out.data_ptr()),
                                       out.shape[1], 1 if accumulate else 0), "qg_learned_apply_d")
        return out

    def gradient(self, grid, R, V, vscale, Y):
        """(loss, gradient) of one batch on the device (FP32 gradient, host)."""
        self._check(grid, R, V, Y=Y)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_double()
        self.ctx.use_torch_stream()
        check(lib().qg_learned_gradient(self.h, grid[0], grid[1], grid[2], R.shape[0], C.c_void_p(R.data_ptr()),
                                        R.shape[1], C.c_void_p(V.data_ptr()), float(vscale), C.c_void_p(Y.data_ptr()),
                                        Y.shape[1], C.byref(loss), g.ctypes.data_as(C.POINTER(C.c_float))),
              "qg_learned_gradient")
        return loss.value, g

    def train_step(self, grid, R, V, vscale, Y, lr):
        self._check(grid, R, V, Y=Y)
        loss = C.c_double()
        self.ctx.use_torch_stream()
        check(lib().qg_learned_train_step(self.h, grid[0], grid[1], grid[2], R.shape[0], C.c_void_p(R.data_ptr()),
                                          R.shape[1], C.c_void_p(V.data_ptr()), float(vscale),
                                          C.c_void_p(Y.data_ptr()), Y.shape[1], float(lr), C.byref(loss)),
              "qg_learned_train_step")
        return loss.value

    def close(self):
        if self.h:
            lib().qg_learned_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Hamiltonian:
    """The device operator H = V + V_NL - 1/2 Lap (qg_hamiltonian).

    ``cell`` is a :class:`qumasun_b200.cell.Cell` (or any object with the same
    fields and ``desc_arrays()``).
    """

    def __init__(self, ctx: Context, cell, fd_order=None, kvec=(0.0, 0.0, 0.0)):
        self.ctx = ctx
        self.cell = cell
        self.N = cell.N
        self._arrays = a = cell.desc_arrays()
        d = HamiltonianDesc()
        d.nx, d.ny, d.nz = cell.nx, cell.ny, cell.nz
        d.hx, d.hy, d.hz = cell.hx, cell.hy, cell.hz
        d.fd_order = int(fd_order if fd_order is not None else cell.fd_order)
        d.V = _ptr(a["V"], _dp)
        npj = len(cell.proj_l)
        d.n_atoms = cell.n_atoms if npj else 0
        d.atom_pos = _ptr(a["atom_pos"], _dp)
        d.n_proj = npj
        d.proj_l = _ptr(a["proj_l"], _ip) if npj else None
        d.proj_E = _ptr(a["proj_E"], _dp) if npj else None
        d.cube = _ptr(a["cube"], _ip)
        d.w_data = _ptr(a["w_data"], _dp)
        d.w_off = _ptr(a["w_off"], _lp)
        d.n_lm = cell.n_lm
        d.ylm_data = _ptr(a["ylm_data"], _dp)
        d.ylm_off = _ptr(a["ylm_off"], _lp)
        d.gx, d.gy, d.gz = kvec
        self.desc = d
        self.h = C.c_void_p()
        check(lib().qg_hamiltonian_create(ctx.h, C.byref(d), C.byref(self.h)), "qg_hamiltonian_create")
        ctx.children.add(self)

    def apply_device(self, ns, x_ptr, hx_ptr, ldx=None, ldhx=None, dtype="f64"):
        """HX = H X on device pointers (int addresses), state-major."""
        ldx = self.N if ldx is None else ldx
        ldhx = self.N if ldhx is None else ldhx
        fn = lib().qg_hamiltonian_apply_d if dtype == "f64" else lib().qg_hamiltonian_apply_f
        check(fn(self.h, ns, C.c_void_p(x_ptr), ldx, C.c_void_p(hx_ptr), ldhx),
              "qg_hamiltonian_apply_" + ("d" if dtype == "f64" else "f"))

    def _check_block(self, X, name, dtypes):
        """A state block the kernels may read or write whole: a contiguous CUDA tensor
        (ns, N) of one of `dtypes` on this context's device."""
        import torch
        if not isinstance(X, torch.Tensor) or not X.is_cuda:
            raise TypeError(f"{name} must be a CUDA tensor")
        if X.dtype not in dtypes:
            raise TypeError(f"{name} has dtype {X.dtype}, expected one of {dtypes}")
        if X.dim() != 2 or X.shape[1] != self.N:
            raise ValueError(f"{name} has shape {tuple(X.shape)}, expected (ns, {self.N})")
        if not X.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
        if X.device.index != self.ctx.device:
            raise ValueError(f"{name} is on cuda:{X.device.index}, the operator on cuda:{self.ctx.device}")

    def apply(self, X, out=None):
        """HX = H X for torch CUDA tensors (ns, N) of float64 or float32."""
        import torch
        self._check_block(X.contiguous() if isinstance(X, torch.Tensor) else X, "X",
                          (torch.float64, torch.float32))
        X = X.contiguous()
        if out is None:
            out = torch.empty_like(X)
        self._check_block(out, "out", (X.dtype,))
        if out.shape != X.shape:
            raise ValueError(f"out has shape {tuple(out.shape)}, X {tuple(X.shape)}")
        dt = "f64" if X.dtype == torch.float64 else "f32"
        self.ctx.use_torch_stream()
        self.apply_device(X.shape[0], X.data_ptr(), out.data_ptr(), dtype=dt)
        return out

    def apply_noalloc(self, X, out):
        """HX = H X (FP64 torch CUDA tensors) through the entry point that allocates
        nothing: the projector coefficients use the library's fixed scratch array.
        X and out must be contiguous float64 CUDA tensors of the same shape (ns, N) on
        the operator's device; anything else raises before the library is called."""
        import torch
        self._check_block(X, "X", (torch.float64,))
        self._check_block(out, "out", (torch.float64,))
        if out.shape != X.shape:
            raise ValueError(f"out has shape {tuple(out.shape)}, X {tuple(X.shape)}")
        self.ctx.use_torch_stream()
        check(lib().qg_hamiltonian_apply_noalloc_d(self.h, X.shape[0], C.c_void_p(X.data_ptr()), self.N,
                                                   C.c_void_p(out.data_ptr()), self.N),
              "qg_hamiltonian_apply_noalloc_d")
        return out

    def lobpcg(self, X0, max_iter=2000, tol=1.0e-10, P0=None, first=True, verbose=False, precond=0,
               shift=1.0):
        """Block LOBPCG (qg_lobpcg_d) from host states X0 (ns, N); returns
        dict(ev, X, P, report, status). NOT_CONVERGED is reported, not raised."""
        X = np.ascontiguousarray(X0, dtype=np.float64).copy()
        ns = X.shape[0]
        P = np.zeros_like(X) if P0 is None else np.ascontiguousarray(P0, dtype=np.float64).copy()
        ev = np.zeros(ns)
        opt = LobpcgOptions(max_iter, tol, 1 if first else 0, 0, 1 if verbose else 0, precond, shift)
        rep = LobpcgReport()
        st = lib().qg_lobpcg_d(self.h, C.byref(opt), ns, ev.ctypes.data_as(_dp), X.ctypes.data, P.ctypes.data,
                               C.byref(rep))
        if st not in (QG_OK, -9):
            check(st, "qg_lobpcg_d")
        return dict(ev=ev, X=X, P=P, report=rep.as_dict(), status=st)

    def lobpcg_device(self, X, P=None, max_iter=2000, tol=1.0e-10, first=True, verbose=False, precond=0,
                      shift=1.0, complex_states=False, n_converge=0, precision=0):
        """Block LOBPCG on device tensors (float64 CUDA, (ns, N) real or (ns, 2N)
        split-complex): X is overwritten with the eigenvectors, P (same shape, may be
        None on a first call) with the last search directions. Returns dict(ev, report, status)."""
        assert X.is_cuda and X.dtype.is_floating_point and X.is_contiguous()
        ns = X.shape[0]
        ev = np.zeros(ns)
        opt = LobpcgOptions(max_iter, tol, 1 if first else 0, precision, 1 if verbose else 0, precond, shift,
                            n_converge)
        rep = LobpcgReport()
        self.ctx.use_torch_stream()
        fn = lib().qg_lobpcg_z_device if complex_states else lib().qg_lobpcg_d_device
        st = fn(self.h, C.byref(opt), ns, ev.ctypes.data_as(_dp), C.c_void_p(X.data_ptr()),
                C.c_void_p(P.data_ptr() if P is not None else 0), C.byref(rep))
        if st not in (QG_OK, -9):
            check(st, "qg_lobpcg_z_device" if complex_states else "qg_lobpcg_d_device")
        return dict(ev=ev, report=rep.as_dict(), status=st)

    def lobpcg_zk(self, kvecs, X, P=None, max_iter=2000, tol=1.0e-10, first=True, verbose=False, precond=0,
                  shift=1.0, n_converge=0):
        """Complex LOBPCG for several k-points in one solve: X float64 CUDA tensor
        (nk, nsk, 2N) overwritten with the eigenvectors; returns dict(ev (nk, nsk), report, status)."""
        import torch
        assert X.is_cuda and X.dim() == 3 and X.is_contiguous() and X.dtype == torch.float64
        kv = np.ascontiguousarray(np.asarray(kvecs, dtype=np.float64).reshape(-1, 3))
        nk, nsk = X.shape[0], X.shape[1]
        ev = np.zeros(nk * nsk)
        opt = LobpcgOptions(max_iter, tol, 1 if first else 0, 0, 1 if verbose else 0, precond, shift, n_converge)
        rep = LobpcgReport()
        self.ctx.use_torch_stream()
        st = lib().qg_lobpcg_zk_device(self.h, C.byref(opt), nk, kv.ctypes.data_as(_dp), nsk,
                                       ev.ctypes.data_as(_dp), C.c_void_p(X.data_ptr()),
                                       C.c_void_p(P.data_ptr() if P is not None else 0), C.byref(rep))
        if st not in (QG_OK, -9):
            check(st, "qg_lobpcg_zk_device")
        return dict(ev=ev.reshape(nk, nsk), report=rep.as_dict(), status=st)

    def lobpcg_z(self, X0, max_iter=2000, tol=1.0e-10, P0=None, first=True, verbose=False, precond=0,
                 shift=1.0):
        """Complex block LOBPCG (qg_lobpcg_z) for the k-point operator from host
        split-complex states X0 (ns, 2N); returns dict(ev, X, P, report, status)."""
        X = np.ascontiguousarray(X0, dtype=np.float64).copy()
        ns = X.shape[0]
        P = np.zeros_like(X) if P0 is None else np.ascontiguousarray(P0, dtype=np.float64).copy()
        ev = np.zeros(ns)
        opt = LobpcgOptions(max_iter, tol, 1 if first else 0, 0, 1 if verbose else 0, precond, shift)
        rep = LobpcgReport()
        st = lib().qg_lobpcg_z(self.h, C.byref(opt), ns, ev.ctypes.data_as(_dp), X.ctypes.data, P.ctypes.data,
                               C.byref(rep))
        if st not in (QG_OK, -9):
            check(st, "qg_lobpcg_z")
        return dict(ev=ev, X=X, P=P, report=rep.as_dict(), status=st)

    def apply_timed(self, ns, x_ptr, hx_ptr):
        """FP64 apply with device phase times (ms): (projection, stencil + V, scatter)."""
        ph = (C.c_float * 3)()
        check(lib().qg_hamiltonian_apply_timed_d(self.h, ns, C.c_void_p(x_ptr), self.N,
                                                 C.c_void_p(hx_ptr), self.N, ph),
              "qg_hamiltonian_apply_timed_d")
        return tuple(ph)

    # ---- complex k-point operator: states are (ns, 2N) rows {re[N], im[N]}
    def td_taylor4(self, X, dt):
        """One Taylor-4 propagation step of {re, im} states X (CUDA float64 (ns, 2N), in place)."""
        import torch
        if not (X.is_cuda and X.dtype == torch.float64 and X.is_contiguous() and X.dim() == 2
                and X.shape[1] == 2 * self.N):
            raise TypeError(f"X must be a contiguous float64 CUDA tensor (ns, {2 * self.N})")
        self.ctx.use_torch_stream()
        check(lib().qg_td_taylor4_z(self.h, X.shape[0], float(dt), _dev(X), X.shape[1]), "qg_td_taylor4_z")
        return X

    def nonlocal_force(self, X, occ, forces=None):
        """(forces (na, 3), e_state (ns,), EV) of real states X (CUDA float64 (ns, N))."""
        import torch
        self._check_block(X, "X", (torch.float64,))
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        na = self.cell.n_atoms if len(self.cell.proj_l) else 0
        f = np.zeros(3 * na) if forces is None else np.ascontiguousarray(forces, dtype=np.float64).reshape(-1).copy()
        e = np.zeros(X.shape[0])
        ev = C.c_double()
        self.ctx.use_torch_stream()
        check(lib().qg_nonlocal_force_d(self.h, X.shape[0], _dev(X), X.shape[1], occ.ctypes.data_as(_dp),
                                        f.ctypes.data_as(_dp), e.ctypes.data_as(_dp), C.byref(ev)),
              "qg_nonlocal_force_d")
        return f.reshape(na, 3), e, ev.value

    def set_kvector(self, g):
        check(lib().qg_hamiltonian_set_kvector(self.h, float(g[0]), float(g[1]), float(g[2])),
              "qg_hamiltonian_set_kvector")

    def apply_z(self, X, out=None):
        """H_k X for a torch CUDA tensor (ns, 2N) of split-complex states: float64
        (complex128 states) or float32 (complex64 states)."""
        import torch
        assert X.is_cuda and X.dim() == 2 and X.shape[1] == 2 * self.N
        assert X.dtype in (torch.float64, torch.float32)
        X = X.contiguous()
        if out is None:
            out = torch.empty_like(X)
        self.ctx.use_torch_stream()
        fn, name = ((lib().qg_hamiltonian_apply_z, "qg_hamiltonian_apply_z") if X.dtype == torch.float64
                    else (lib().qg_hamiltonian_apply_zf, "qg_hamiltonian_apply_zf"))
        check(fn(self.h, X.shape[0], C.c_void_p(X.data_ptr()), 2 * self.N, C.c_void_p(out.data_ptr()), 2 * self.N),
              name)
        return out

    def apply_zk(self, kvecs, X, out=None):
        """H_k X for several k-points in one pass: X float64 CUDA tensor (nk, nsk, 2N),
        kvecs (nk, 3) Bloch vectors in bohr^-1."""
        import torch
        assert X.is_cuda and X.dim() == 3 and X.shape[2] == 2 * self.N
        assert X.dtype in (torch.float64, torch.float32)
        X = X.contiguous()
        kv = np.ascontiguousarray(np.asarray(kvecs, dtype=np.float64).reshape(-1, 3))
        assert kv.shape[0] == X.shape[0]
        if out is None:
            out = torch.empty_like(X)
        self.ctx.use_torch_stream()
        nk, nsk = X.shape[0], X.shape[1]
        fn, name = ((lib().qg_hamiltonian_apply_zk, "qg_hamiltonian_apply_zk") if X.dtype == torch.float64
                    else (lib().qg_hamiltonian_apply_zkf, "qg_hamiltonian_apply_zkf"))
        check(fn(self.h, nk, kv.ctypes.data_as(_dp), nsk, C.c_void_p(X.data_ptr()), 2 * self.N, nsk * 2 * self.N,
                 C.c_void_p(out.data_ptr()), 2 * self.N, nsk * 2 * self.N), name)
        return out

    def apply_host_z(self, X: np.ndarray, out: np.ndarray | None = None):
        """H_k X with host buffers (ns, 2N)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        if out is None:
            out = np.empty_like(X)
        check(lib().qg_hamiltonian_apply_host_z(self.h, X.shape[0], X.ctypes.data, out.ctypes.data),
              "qg_hamiltonian_apply_host_z")
        return out

    def apply_timed_z(self, ns, x_ptr, hx_ptr):
        ph = (C.c_float * 3)()
        check(lib().qg_hamiltonian_apply_timed_z(self.h, ns, C.c_void_p(x_ptr), 2 * self.N,
                                                 C.c_void_p(hx_ptr), 2 * self.N, ph),
              "qg_hamiltonian_apply_timed_z")
        return tuple(ph)

    def precondition(self, R, shift=1.0):
        """R <- T R in place (kinetic preconditioner) for a float64 CUDA tensor (ns, N)."""
        self.ctx.use_torch_stream()
        check(lib().qg_hamiltonian_precondition_d(self.h, R.shape[0], C.c_void_p(R.data_ptr()), R.shape[1],
                                                  float(shift)), "qg_hamiltonian_precondition_d")
        return R

    def set_learned(self, nn, vscale=4.0):
        """Attach a LearnedPreconditioner for LOBPCG precond=2 (None detaches)."""
        check(lib().qg_hamiltonian_set_learned(self.h, nn.h if nn is not None else None, float(vscale)),
              "qg_hamiltonian_set_learned")

    def set_stencil_kernel(self, variant):
        """Stencil kernel of the real-state apply: 0 (or False) = engine's choice, 1 (or
        True) = register-window kernel, 2 = one-plane TMA ring, 3 = two-plane TMA ring,
        4 = two rows per thread with V in the ring."""
        v = int(variant)
        check(lib().qg_hamiltonian_set_stencil_kernel(self.h, v), "qg_hamiltonian_set_stencil_kernel")

    def set_nonlocal_blocking(self, project_states=0, scatter_states=0, project_parts=0):
        """States per projection block (1/2/4/8/16), per scatter group (4/8) and blocks per
        atom in the projection (1-8); 0 = engine's choice."""
        check(lib().qg_hamiltonian_set_nonlocal_blocking(self.h, project_states, scatter_states, project_parts),
              "qg_hamiltonian_set_nonlocal_blocking")

    def autotune(self, X, out=None):
        """Times the bit-identical launch shapes on the CUDA block X (float64 or float32,
        (ns, N)) and keeps the fastest; returns dict(stencil, project_states,
        scatter_states, ms_phases)."""
        import torch
        self._check_block(X, "X", (torch.float64, torch.float32))
        out = torch.empty_like(X) if out is None else out
        self._check_block(out, "out", (X.dtype,))
        choice = (C.c_int * 3)()
        ms = (C.c_float * 3)()
        fn = lib().qg_hamiltonian_autotune_d if X.dtype == torch.float64 else lib().qg_hamiltonian_autotune_f
        self.ctx.use_torch_stream()
        check(fn(self.h, X.shape[0], _dev(X), X.shape[1], _dev(out), out.shape[1], choice, ms),
              "qg_hamiltonian_autotune")
        return dict(stencil=choice[0], project_states=choice[1], scatter_states=choice[2],
                    ms_phases=[round(float(v), 4) for v in ms])

    def set_gram_reuse(self, on: bool):
        """Steady-state Gram pencil from the previous rotation (True, default) or a full Gram every step."""
        check(lib().qg_hamiltonian_set_gram_reuse(self.h, 1 if on else 0), "qg_hamiltonian_set_gram_reuse")

    def launches_per_apply(self, ns):
        return lib().qg_hamiltonian_launches_per_apply(self.h, ns)

    def apply_host(self, X: np.ndarray, out: np.ndarray | None = None):
        """HX = H X with host buffers (copies in and out inside the call)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        if out is None:
            out = np.empty_like(X)
        check(lib().qg_hamiltonian_apply_host_d(self.h, X.shape[0], X.ctypes.data, out.ctypes.data),
              "qg_hamiltonian_apply_host_d")
        return out

    def apply_host_ptr(self, ns, x_ptr, hx_ptr):
        check(lib().qg_hamiltonian_apply_host_d(self.h, ns, C.c_void_p(x_ptr), C.c_void_p(hx_ptr)),
              "qg_hamiltonian_apply_host_d")

    def close(self):
        if self.h:
            lib().qg_hamiltonian_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
