"""CPU oracle for the H|psi> + LOBPCG path -- TEST INFRASTRUCTURE ONLY.

Two checkers, both CPU:

* the *port* (``libqg_oracle.so``, built from ``qg_oracle.c``): this project's
  plain-C restatement of the reference functions, and ``lobpcg_d_multi`` below,
  a numpy restatement of EigenLOBPCG_d_multi (lobpcg_d_multi.h:23-545);
* the *reference* (``_ref/libqumasun_ref.so``): the reference's own headers
  compiled by ``oracle/Makefile``, driven through ``ref_harness.cpp``.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs may
import this package, as the checker or the timed CPU baseline; the product
(``qumasun_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libqg_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqumasun_ref.so")
ADAPTER_SO = os.path.join(HERE, "_ref", "libadapter_check.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_longlong)


class HamDescC(C.Structure):
    """Mirror of ref_ham_desc (ref_harness.cpp) / or_ham_desc (qg_oracle.c)."""

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
    ]


def _ptr(a, t):
    return a.ctypes.data_as(t)


class HamDesc:
    """Holds the flat cube-table arrays of a Cell alive behind a HamDescC."""

    def __init__(self, cell, fd_order=None):
        self.arrays = cell.desc_arrays()
        a = self.arrays
        d = HamDescC()
        d.nx, d.ny, d.nz = cell.nx, cell.ny, cell.nz
        d.hx, d.hy, d.hz = cell.hx, cell.hy, cell.hz
        d.fd_order = int(fd_order if fd_order is not None else cell.fd_order)
        d.V = _ptr(a["V"], _dp)
        d.n_atoms = cell.n_atoms if len(cell.proj_l) else 0
        d.atom_pos = _ptr(a["atom_pos"], _dp)
        d.n_proj = len(cell.proj_l)
        d.proj_l = _ptr(a["proj_l"], _ip) if d.n_proj else None
        d.proj_E = _ptr(a["proj_E"], _dp) if d.n_proj else None
        d.cube = _ptr(a["cube"], _ip)
        d.w_data = _ptr(a["w_data"], _dp)
        d.w_off = _ptr(a["w_off"], _lp)
        d.n_lm = cell.n_lm
        d.ylm_data = _ptr(a["ylm_data"], _dp)
        d.ylm_off = _ptr(a["ylm_off"], _lp)
        self.c = d


_port = None
_ref = None


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            raise FileNotFoundError(f"{PORT_SO} missing: run `make -C oracle port`")
        lib = C.CDLL(PORT_SO)
        lib.or_laplacian.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.c_double, _dp, _dp]
        lib.or_laplacian_kpoint8.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                             C.c_double, C.c_double, C.c_double, C.c_double,
                                             C.c_double, _dp, _dp, _dp, _dp]
        lib.or_hamiltonian_apply.argtypes = [C.POINTER(HamDescC), C.c_int, _dp, _dp]
        lib.or_laplacian_kpoint.argtypes = [C.c_int] * 4 + [C.c_double] * 7 + [_dp] * 4
        lib.or_hamiltonian_kpoint_local.argtypes = [C.POINTER(HamDescC), C.c_double, C.c_double,
                                                    C.c_double, C.c_int, _dp, _dp]
        lib.or_hamiltonian_kpoint_apply.argtypes = [C.POINTER(HamDescC), C.c_double, C.c_double,
                                                    C.c_double, C.c_int, _dp, _dp]
        _port = lib
    return _port


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing: run `make -C oracle ref` where the reference tree exists")
        lib = C.CDLL(REF_SO)
        lib.ref_laplacian.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                      C.c_double, C.c_double, _dp, _dp]
        lib.ref_laplacian_kpoint8.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                              C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_double, _dp, _dp, _dp, _dp]
        lib.ref_hamiltonian_apply.argtypes = [C.POINTER(HamDescC), C.c_int, _dp, _dp]
        lib.ref_laplacian_kpoint.argtypes = [C.c_int] * 4 + [C.c_double] * 7 + [_dp] * 4
        lib.ref_lobpcg_d_multi.argtypes = [C.POINTER(HamDescC), C.c_int, C.c_int, _dp, _dp, _dp,
                                           C.c_int, C.c_int, _ip]
        lib.ref_grid_for_sphere.argtypes = [C.c_double] * 7 + [_ip]
        lib.ref_ylm_cube.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp]
        lib.ref_hamiltonian_kpoint_apply.argtypes = [C.POINTER(HamDescC), C.c_double, C.c_double,
                                                     C.c_double, C.c_double, C.c_int, _dp, _dp]
        lib.ref_lobpcg_d_mpi.argtypes = [C.POINTER(HamDescC), C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_int,
                                         _dp, _dp, _ip]
        lib.ref_lobpcg_z_multi.argtypes = [C.POINTER(HamDescC), C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.c_int, C.c_int, _dp, _dp, C.c_int, _ip]
        lib.ref_potential_lda.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [_dp] * 7
        lib.ref_set_occupancy.argtypes = [C.c_double, C.c_double, C.c_int, _dp, C.c_double, _dp]
        lib.ref_set_occupancy.restype = C.c_double
        lib.ref_gradient8.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [_dp] * 4
        lib.ref_td_taylor4.argtypes = [C.POINTER(HamDescC)] + [C.c_double] * 5 + [C.c_int, _dp]
        lib.ref_nonlocal_force_z.argtypes = [C.POINTER(HamDescC)] + [C.c_double] * 4 + [C.c_int, _dp, _dp, _dp,
                                                                                          _dp, _dp]
        lib.ref_nonlocal_energy_d.argtypes = [C.POINTER(HamDescC), C.c_int, _dp, _dp]
        _ref = lib
    return _ref


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------- stencils
def laplacian(order, grid, h, coef, psi, impl="port"):
    """out = coef * Lap(psi) for one state (starting from zeros)."""
    nx, ny, nz = grid
    psi = _c64(psi)
    out = np.zeros_like(psi)
    lib = port_lib() if impl == "port" else ref_lib()
    fn = lib.or_laplacian if impl == "port" else lib.ref_laplacian
    rc = fn(order, nx, ny, nz, h[0], h[1], h[2], coef, _ptr(psi, _dp), _ptr(out, _dp))
    if rc != 0:
        raise ValueError(f"laplacian order {order} rejected ({rc})")
    return out


def laplacian_kpoint(order, grid, h, coef, g, re, im, impl="port"):
    """(out_re, out_im) += coef (Lap + 2i g.grad - g^2) on split re/im arrays, FD order 2,
    6 or 8 (LaplasianKpoint{2nd,6th,8th}_halo)."""
    lib = port_lib() if impl == "port" else ref_lib()
    fn = lib.or_laplacian_kpoint if impl == "port" else lib.ref_laplacian_kpoint
    re, im = _c64(re), _c64(im)
    ore, oim = np.zeros_like(re), np.zeros_like(im)
    rc = fn(order, grid[0], grid[1], grid[2], h[0], h[1], h[2], coef, g[0], g[1], g[2], _ptr(re, _dp), _ptr(im, _dp),
            _ptr(ore, _dp), _ptr(oim, _dp))
    if rc != 0:
        raise ValueError(f"laplacian_kpoint rejected order {order}")
    return ore, oim


def laplacian_kpoint8(grid, h, coef, g, re, im, impl="port"):
    nx, ny, nz = grid
    re, im = _c64(re), _c64(im)
    ore, oim = np.zeros_like(re), np.zeros_like(im)
    lib = port_lib() if impl == "port" else ref_lib()
    fn = lib.or_laplacian_kpoint8 if impl == "port" else lib.ref_laplacian_kpoint8
    fn(nx, ny, nz, h[0], h[1], h[2], coef, g[0], g[1], g[2], _ptr(re, _dp), _ptr(im, _dp),
       _ptr(ore, _dp), _ptr(oim, _dp))
    return ore, oim


# ------------------------------------------------------------- Hamiltonian
def hamiltonian_apply(cell, X, impl="port", fd_order=None):
    """HX = H X for a state-major block X (ns, N), FP64."""
    X = _c64(X)
    ns = X.shape[0]
    HX = np.zeros_like(X)
    desc = HamDesc(cell, fd_order)
    if impl == "port":
        rc = port_lib().or_hamiltonian_apply(C.byref(desc.c), ns, _ptr(X, _dp), _ptr(HX, _dp))
    else:
        rc = ref_lib().ref_hamiltonian_apply(C.byref(desc.c), ns, _ptr(X, _dp), _ptr(HX, _dp))
    if rc != 0:
        raise ValueError(f"hamiltonian_apply rejected ({rc})")
    return HX


def hamiltonian_kpoint_local(cell, g, X):
    """Local part (V + k-point kinetic) of the complex H on {re, im} states (ns, 2N)."""
    X = _c64(X)
    HX = np.zeros_like(X)
    desc = HamDesc(cell, 8)
    port_lib().or_hamiltonian_kpoint_local(C.byref(desc.c), g[0], g[1], g[2], X.shape[0],
                                           _ptr(X, _dp), _ptr(HX, _dp))
    return HX


def hamiltonian_kpoint_apply(cell, g, X, impl="port", fd_order=8):
    """Complex k-point H (V + nonlocal with Bloch phases + 8th-order k-point kinetic)
    on {re, im} states X (ns, 2N); g = Bloch vector in bohr^-1."""
    X = _c64(X)
    HX = np.zeros_like(X)
    desc = HamDesc(cell, fd_order)
    if impl == "port":
        rc = port_lib().or_hamiltonian_kpoint_apply(C.byref(desc.c), g[0], g[1], g[2], X.shape[0],
                                                    _ptr(X, _dp), _ptr(HX, _dp))
    else:
        rc = ref_lib().ref_hamiltonian_kpoint_apply(C.byref(desc.c), g[0], g[1], g[2], cell.cutoff,
                                                    X.shape[0], _ptr(X, _dp), _ptr(HX, _dp))
    if rc != 0:
        raise ValueError(f"hamiltonian_kpoint_apply rejected ({rc})")
    return HX


# ------------------------------------------------------------------ LOBPCG
def ref_lobpcg_d_multi(cell, X0, iter_max, P0=None, first=True, quiet=True):
    """The reference's EigenLOBPCG_d_multi run unchanged (X0 is not modified)."""
    X = _c64(X0).copy()
    ns = X.shape[0]
    P = np.zeros_like(X) if P0 is None else _c64(P0).copy()
    ev = np.zeros(ns)
    iters = C.c_int(0)
    desc = HamDesc(cell)
    t0 = time.perf_counter()
    ref_lib().ref_lobpcg_d_multi(C.byref(desc.c), ns, iter_max, _ptr(ev, _dp), _ptr(X, _dp),
                                 _ptr(P, _dp), 1 if first else 0, 1 if quiet else 0,
                                 C.byref(iters))
    return dict(ev=ev, X=X, P=P, iters=iters.value, seconds=time.perf_counter() - t0)


def ref_lobpcg_d_mpi(cell, X0, iter_max, threads=8, quiet=True, in_place=False):
    """The reference's distributed real solver LOBPCG::Eigen_d_multi_mpi
    (lobpcg_d_multi_mpi.h:882-1572) on one rank, SCF step 0, DGEMMs on `threads`
    OpenBLAS threads. X0 (ns, N) is left unchanged unless in_place (then it must be a
    C-contiguous float64 array and receives the states; no copy is made). Returns the
    eigenvalues, states, iterations, the phase seconds (H applications, Gram, rotation,
    n x n GEMMs, small eigensolve, rest, total) of the reference's own watch sections
    and the seconds of each iteration."""
    X = X0 if in_place else _c64(X0).copy()
    if in_place and (X.dtype != np.float64 or not X.flags.c_contiguous):
        raise ValueError("in_place needs a C-contiguous float64 array")
    ns = X.shape[0]
    ev = np.zeros(ns)
    ph = np.zeros(7)
    its = np.zeros(max(1, iter_max))
    iters = C.c_int(0)
    desc = HamDesc(cell)
    ref_lib().ref_lobpcg_d_mpi(C.byref(desc.c), ns, iter_max, threads, _ptr(ev, _dp), _ptr(X, _dp),
                               1 if quiet else 0, _ptr(ph, _dp), _ptr(its, _dp), C.byref(iters))
    names = ("hamiltonian", "gram", "rotation", "small_gemm", "eigensolve", "rest", "total")
    return dict(ev=ev, X=X, iters=iters.value, phase_s={k: float(v) for k, v in zip(names, ph)},
                iteration_s=[float(v) for v in its[:iter_max]])


def ref_lobpcg_z_multi(cell, g, X0, iter_max, quiet=True):
    """The reference's complex Eigen_z_multi_mpi (one rank, SCF step 0) with the reference
    k-point H; X0 (ns, 2N) {re, im} states is not modified."""
    X = _c64(X0).copy()
    ns = X.shape[0]
    ev = np.zeros(ns)
    iters = C.c_int(0)
    desc = HamDesc(cell, 8)
    t0 = time.perf_counter()
    rc = ref_lib().ref_lobpcg_z_multi(C.byref(desc.c), g[0], g[1], g[2], cell.cutoff, ns, iter_max,
                                      _ptr(ev, _dp), _ptr(X, _dp), 1 if quiet else 0, C.byref(iters))
    if rc != 0:
        raise ValueError(f"ref_lobpcg_z_multi rejected ({rc})")
    return dict(ev=ev, X=X, iters=iters.value, seconds=time.perf_counter() - t0)


def dense_kpoint_hamiltonian(cell, g):
    """The k-point H of the port as a dense complex N x N matrix (small grids only):
    column j is H_k applied to the j-th unit vector."""
    N = cell.N
    H = np.zeros((N, N), dtype=np.complex128)
    blk = 256
    for j0 in range(0, N, blk):
        j1 = min(N, j0 + blk)
        X = np.zeros((j1 - j0, 2 * N))
        X[np.arange(j1 - j0), np.arange(j0, j1)] = 1.0
        HX = hamiltonian_kpoint_apply(cell, g, X)
        H[:, j0:j1] = (HX[:, :N] + 1j * HX[:, N:]).T
    return H


def lobpcg_d_multi(apply_H, X0, dV, iter_max, limit=1.0e-10, P0=None, first=True, callback=None):
    """numpy restatement of EigenLOBPCG_d_multi (lobpcg_d_multi.h:23-545).

    Same steps, with the scalar InnerProd / AddV loops written as block
    products: normalise x (Normalize, vecmath.h:128), r = Ax - (x.Ax dV) x
    normalised (:64-91); per iteration Ar = H r, the 3n x 3n pencil
    (Sa, Sb) = ([x r p]^T [Ax Ar Ap], [x r p]^T [x r p]) * dV (:103-133), the
    2n x 2n (x, r) pencil on the very first step (:157-235), the generalised
    eigensolve with LAPACK dsygvx (RANGE=A, UPLO=U, ABSTOL=1e-13,
    w_dsygvx.h:24-104), the rotation P = R Cr + P Cp, X = X Cx + P (:247-300),
    renormalisation of x, p, Ax, Ap (:491-505), the Rayleigh quotient and the
    residual exit max(sum r^2 dV) < limit dV (:506-525).
    ``apply_H`` maps a state-major (ns, N) block to H times it.
    """
    import scipy.linalg as sl

    x = _c64(X0).copy()
    n = x.shape[0]
    x /= np.sqrt(np.einsum("ij,ij->i", x, x) * dV)[:, None]
    p = np.zeros_like(x) if (P0 is None or first) else _c64(P0).copy()
    Ax = apply_H(x)
    Ap = np.zeros_like(x) if first else apply_H(p)
    ei = np.einsum("ij,ij->i", x, Ax) * dV
    r = Ax - ei[:, None] * x
    r /= np.sqrt(np.einsum("ij,ij->i", r, r) * dV)[:, None]
    it = 0
    history = []
    for it in range(iter_max):
        Ar = apply_H(r)
        first_step = first and it == 0
        if first_step:
            V = np.concatenate([x, r])
            AV = np.concatenate([Ax, Ar])
        else:
            V = np.concatenate([x, r, p])
            AV = np.concatenate([Ax, Ar, Ap])
        Sa = (V @ AV.T) * dV
        Sb = (V @ V.T) * dV
        w, Z = sl.eigh(Sa, Sb, lower=False, driver="gvx")
        Cx, Cr = Z[:n, :n], Z[n:2 * n, :n]
        if first_step:
            p = Cr.T @ r
            Ap = Cr.T @ Ar
        else:
            Cp = Z[2 * n:, :n]
            p = Cr.T @ r + Cp.T @ p
            Ap = Cr.T @ Ar + Cp.T @ Ap
        x = Cx.T @ x + p
        Ax = Cx.T @ Ax + Ap
        nx_ = 1.0 / np.sqrt(np.einsum("ij,ij->i", x, x) * dV)
        np_ = 1.0 / np.sqrt(np.einsum("ij,ij->i", p, p) * dV)
        x *= nx_[:, None]
        Ax *= nx_[:, None]
        p *= np_[:, None]
        Ap *= np_[:, None]
        ei = np.einsum("ij,ij->i", x, Ax) * dV
        r = Ax - ei[:, None] * x
        norm_r = np.einsum("ij,ij->i", r, r) * dV
        history.append(float(norm_r.max()))
        if callback is not None:
            callback(it, ei, norm_r)
        if norm_r.max() < limit * dV:
            break
    return dict(ev=ei, X=x, P=p, iters=it + 1 if iter_max > 0 else 0, history=history)


# ---------------------------------------------------------------- SCF-step neighbours
# Reference entry points (oracle/_ref) and numpy restatements (the port) of the
# density, occupations, Poisson + LDA potential, Taylor-4 propagation and nonlocal
# energy/forces. The restatements follow the cited reference lines; the tests pin
# them against the reference harness.

def density(X, occ, rho0=None):
    """rho = rho0 + sum_s occ[s] * X[s]^2 over occ > 0, states in order, each term
    (p*p)*f added (QUMASUN_SINGLE::mSetDensityOne, qumasun_single.density.h:10-27)."""
    X = _c64(X)
    rho = np.zeros(X.shape[1]) if rho0 is None else np.array(rho0, dtype=np.float64)
    for s in range(X.shape[0]):
        if occ[s] <= 0.0:
            continue
        rho += (X[s] * X[s]) * occ[s]
    return rho


def density_z(X, occ, rho0=None):
    """Complex {re, im} states (ns, 2N): rho += (re*re + im*im) * f
    (QUMASUN_KPOINT::mSetDensityOne, qumasun_kpoint.density.h:11-33)."""
    X = _c64(X)
    N = X.shape[1] // 2
    rho = np.zeros(N) if rho0 is None else np.array(rho0, dtype=np.float64)
    for s in range(X.shape[0]):
        if occ[s] <= 0.0:
            continue
        re, im = X[s, :N], X[s, N:]
        rho += (re * re + im * im) * occ[s]
    return rho


def fermi(coef, kbT, ev, mu, impl="port"):
    """Occupations at chemical potential mu and their sum (SetOccupancy.h:7-18)."""
    ev = _c64(ev)
    if impl == "ref":
        occ = np.zeros_like(ev)
        tot = ref_lib().ref_set_occupancy(coef, kbT, len(ev), _ptr(ev, _dp), mu, _ptr(occ, _dp))
        return occ, tot
    p = np.minimum((1.0 / kbT) * (ev - mu), 80.0)
    occ = coef / (np.exp(p) + 1.0)
    tot = 0.0
    for v in occ:
        tot += v
    return occ, tot


def occupancy(kbT, ev, n_electrons, impl="port"):
    """Bisection on mu of QUMASUN_SINGLE::mSetOccupancySpinOff (qumasun_single.occupancy.h:19-55)
    around SetOccupancy (the reference's own function with impl='ref')."""
    ev = _c64(ev)
    n = len(ev)
    mu_min, mu_max = ev[0], ev[n - 1]
    mu_max = mu_max * 16.0 if mu_max > 0.0 else abs(mu_max) + 16.0
    if (n_electrons + 1) // 2 >= n:
        mu_max *= 10.0
    mu = (mu_min + mu_max) / 2.0
    occ = np.zeros(n)
    while abs(mu_max - mu_min) > 1.0e-9:
        occ, num_e = fermi(2.0, kbT, ev, mu, impl)
        if num_e < n_electrons:
            mu_min = mu
        elif num_e > n_electrons:
            mu_max = mu
        else:
            break
        mu = (mu_min + mu_max) / 2.0
    return occ, mu


def potential_lda(grid, h, rho, vext, pcc=None, impl="ref"):
    """(vtot, vhart, vx, vc) of QUMASUN_SINGLE::mSetPotential for KohnSham_PP without spin.
    impl='ref': the reference's SetPotentialByPoissonFFT (poisson_fft.h:14-128, FFTW
    supplied by shims/fftw3.h) and Calc_XC_LDA (Vxc.h:41-70); impl='port': numpy FFT."""
    nx, ny, nz = grid
    rho = _c64(rho)
    vext = _c64(vext)
    N = nx * ny * nz
    if impl == "ref":
        out = [np.zeros(N) for _ in range(4)]
        pc = _c64(pcc) if pcc is not None else None
        ref_lib().ref_potential_lda(nx, ny, nz, h[0], h[1], h[2], _ptr(rho, _dp),
                                    _ptr(pc, _dp) if pc is not None else None, _ptr(vext, _dp),
                                    *[_ptr(o, _dp) for o in out])
        return tuple(out)
    rk = np.fft.fftn(rho.reshape(nz, ny, nx))
    def fold(n, hh):
        k = np.arange(n)
        return (2.0 * np.pi / (hh * n)) * np.where(k < n // 2, k, k - n)
    kx, ky, kz = fold(nx, h[0]), fold(ny, h[1]), fold(nz, h[2])
    k2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    scale = 4.0 * np.pi / k2
    scale[0, 0, 0] = 0.0
    vh = np.fft.ifftn(rk * scale).real.reshape(-1)
    r = rho + (_c64(pcc) if pcc is not None else 0.0)
    vx, vc = lda_pz81(r)
    return vext + vh + vx + vc, vh, vx, vc


def lda_pz81(rho):
    """Perdew-Zunger 1981 LDA potentials (V_x, V_c) of an unpolarised density, as
    Calc_XC_LDA (Vxc.h:41-70) forms them; zero below 1e-8."""
    rho = np.asarray(rho, dtype=np.float64)
    vx = np.zeros_like(rho)
    vc = np.zeros_like(rho)
    m = rho >= 1.0e-8
    c2 = np.cbrt(3.0 / (4.0 * np.pi))
    c3 = -(3.0 / (4.0 * np.pi)) * np.cbrt(9.0 * np.pi / 4.0)
    rs = c2 / np.cbrt(rho[m])
    ex0 = c3 / rs
    ge = rs >= 1.0
    ec = np.empty_like(rs)
    ndec = np.empty_like(rs)
    sq = np.sqrt(rs[ge])
    g, b1, b2 = -0.1423, 1.0529, 0.3334
    ec[ge] = g / (1.0 + b1 * sq + b2 * rs[ge])
    ndec[ge] = ec[ge] * ec[ge] * (b1 * 0.5 * sq + b2 * rs[ge]) / (3.0 * g)
    lt = ~ge
    A, B, Cc, D = 0.0311, -0.0480, 0.0020, -0.0116
    lr = np.log(rs[lt])
    ec[lt] = B + A * lr + D * rs[lt] + Cc * rs[lt] * lr
    ndec[lt] = -(A + (D + Cc) * rs[lt] + Cc * rs[lt] * lr) / 3.0
    vx[m] = ex0 + ex0 / 3.0
    vc[m] = ec + ndec
    return vx, vc


def gradient8(grid, h, coef, psi, impl="port"):
    """coef * grad psi, 8th order, periodic (Gradient8th, GridGradient8th.h:19-235)."""
    nx, ny, nz = grid
    psi = _c64(psi)
    if impl == "ref":
        out = [np.zeros(nx * ny * nz) for _ in range(3)]
        ref_lib().ref_gradient8(nx, ny, nz, h[0], h[1], h[2], coef, _ptr(psi, _dp), *[_ptr(o, _dp) for o in out])
        return out
    p = psi.reshape(nz, ny, nx)
    out = []
    for ax, hh in zip((2, 1, 0), h):
        c = [k * coef / (840.0 * hh) for k in (672.0, -168.0, 32.0, -3.0)]
        d = [np.roll(p, -s, axis=ax) - np.roll(p, s, axis=ax) for s in (1, 2, 3, 4)]
        out.append((c[3] * d[3] + c[2] * d[2] + c[1] * d[1] + c[0] * d[0]).reshape(-1))
    return out


def td_taylor4(cell, g, dt, X, impl="ref"):
    """One Taylor-4 step of {re, im} states (ns, 2N) under the k-point H at Bloch vector g.
    impl='ref': QUMASUN::TimeEvoH4 (qumasun_td.time_evo_H4.h:13-60) run unchanged with the
    reference's k-point H; impl='port': the same update sequence around the port's H."""
    X = _c64(X).copy()
    if impl == "ref":
        desc = HamDesc(cell, 8)
        rc = ref_lib().ref_td_taylor4(C.byref(desc.c), g[0], g[1], g[2], cell.cutoff, dt, X.shape[0], _ptr(X, _dp))
        if rc != 0:
            raise ValueError(f"ref_td_taylor4 rejected ({rc})")
        return X
    N = X.shape[1] // 2
    c2 = dt * dt / 2.0
    c3 = c2 * dt / 3.0
    c4 = c3 * dt / 4.0
    H1 = hamiltonian_kpoint_apply(cell, g, X)
    X[:, :N] += dt * H1[:, N:]
    X[:, N:] += -dt * H1[:, :N]
    H2 = hamiltonian_kpoint_apply(cell, g, H1)
    X += -c2 * H2
    H3 = hamiltonian_kpoint_apply(cell, g, H2)
    X[:, :N] += -c3 * H3[:, N:]
    X[:, N:] += c3 * H3[:, :N]
    H4 = hamiltonian_kpoint_apply(cell, g, H3)
    X += c4 * H4
    return X


def nonlocal_force(cell, X, occ, g=(0.0, 0.0, 0.0), impl="ref"):
    """(forces (na, 3), e_state (ns,), EV) of the nonlocal pseudopotential.
    X: real states (ns, N) or complex {re, im} states (ns, 2N).
    impl='ref': the reference's Gradient8th + PseudoPotIntegrator_kpoint::ForceNonlocal
    (PseudoPotOperator_kpoint_v2.h:2760-2866) per occupied state, as
    mGetForcePseudoNonlocal (qumasun_kpoint.force.h:238-258) calls them;
    impl='port': numpy inner products over the cube tables (Gamma, real states)."""
    X = _c64(X)
    N = cell.N
    ns = X.shape[0]
    cplx = X.shape[1] == 2 * N
    na = cell.n_atoms
    if impl == "ref":
        Z = X if cplx else np.concatenate([X, np.zeros_like(X)], axis=1)
        Z = np.ascontiguousarray(Z)
        desc = HamDesc(cell, 8)
        forces = np.zeros(3 * na)
        e = np.zeros(ns)
        ev = np.zeros(1)
        oc = _c64(occ)
        rc = ref_lib().ref_nonlocal_force_z(C.byref(desc.c), g[0], g[1], g[2], cell.cutoff, ns, _ptr(Z, _dp),
                                            _ptr(oc, _dp), _ptr(forces, _dp), _ptr(e, _dp), _ptr(ev, _dp))
        if rc != 0:
            raise ValueError(f"ref_nonlocal_force_z rejected ({rc})")
        return forces.reshape(na, 3), e, float(ev[0])
    if cplx:
        raise NotImplementedError("the port covers real states")
    grid = (cell.nx, cell.ny, cell.nz)
    h = (cell.hx, cell.hy, cell.hz)
    forces = np.zeros((na, 3))
    e = np.zeros(ns)
    ev = 0.0
    for s in range(ns):
        inner = _inner_products(cell, X[s])
        e[s] = sum(E * v * v for per in inner for v, E in per)
        if occ[s] <= 0.0:
            continue
        dps = gradient8(grid, h, -2.0 * occ[s], X[s])
        dins = [_inner_products(cell, d) for d in dps]
        for a in range(na):
            for d in range(3):
                forces[a, d] += sum(dv * v * E for (v, E), (dv, _) in zip(inner[a], dins[d][a]))
        ev += e[s] * occ[s]
    return forces, e, ev


def _inner_products(cell, psi):
    """Per atom, the list of (dV <w_k Y_lm | psi>, E_k) over projectors k and m
    (InnerProd_1S_1R / InnerProd_2S_1R of EnergyPPnonlocal, PseudoPotOperator.h:775-816)."""
    nx, ny, nz = cell.nx, cell.ny, cell.nz
    p = psi.reshape(nz, ny, nx)
    y00 = 1.0 / np.sqrt(4.0 * np.pi)
    out = []
    for a in range(cell.n_atoms):
        per = []
        for k, l in enumerate(cell.proj_l):
            b, size, w = cell.cubes[a][k]
            zi = np.arange(b[2], b[2] + size[2]) % nz
            yi = np.arange(b[1], b[1] + size[1]) % ny
            xi = np.arange(b[0], b[0] + size[0]) % nx
            sub = p[np.ix_(zi, yi, xi)].reshape(-1)
            if l == 0:
                per.append((cell.dV * y00 * float(np.dot(w, sub)), cell.proj_E[k]))
            else:
                for m in range(2 * l + 1):
                    y = cell.ylm_tabs[a][l * l + m]
                    per.append((cell.dV * float(np.dot(w * y, sub)), cell.proj_E[k]))
        out.append(per)
    return out


def nonlocal_energy(cell, X):
    """Nonlocal energy of each real state (PseudoPotIntegrator_single::EnergyPPnonlocal,
    PseudoPotOperator.h:775-816), the reference's own function."""
    X = _c64(X)
    e = np.zeros(X.shape[0])
    desc = HamDesc(cell, 8)
    ref_lib().ref_nonlocal_energy_d(C.byref(desc.c), X.shape[0], _ptr(X, _dp), _ptr(e, _dp))
    return e


# ---------------------------------------------------------------- C++ adapter checks
_adapter = None


def adapter_available():
    return os.path.exists(ADAPTER_SO)


def adapter_lib():
    """oracle/_ref/libadapter_check.so: the reference's call sites driving
    include/qumasun_b200_adapter.hpp (adapter_check.cpp)."""
    global _adapter
    if _adapter is None:
        lib = C.CDLL(ADAPTER_SO)
        geo = [C.c_int] * 3 + [C.c_double] * 3 + [C.c_int, _dp, C.c_int, _ip, _dp, C.c_double, C.c_double, _dp]
        lib.adapter_flatten_stats.argtypes = geo + [_ip, _dp]
        lib.adapter_apply_check.argtypes = geo + [C.c_int, _dp, _dp, _dp]
        lib.adapter_lobpcg_check.argtypes = geo + [C.c_int, C.c_int, _dp, _dp, _dp, _ip]
        _adapter = lib
    return _adapter


def _adapter_geo(cell, sigma):
    pos = _c64(cell.positions.reshape(-1))
    pl = np.array(cell.proj_l, dtype=np.int32)
    pe = np.array(cell.proj_E, dtype=np.float64)
    V = _c64(cell.V)
    keep = (pos, pl, pe, V)
    args = [cell.nx, cell.ny, cell.nz, cell.hx, cell.hy, cell.hz, cell.n_atoms, _ptr(pos, _dp), len(pl),
            _ptr(pl, _ip), _ptr(pe, _dp), cell.cutoff, sigma, _ptr(V, _dp)]
    return keep, args


def adapter_flatten_stats(cell, sigma):
    """(code, cubes (na*np, 6), sums [flattened w, direct w, flattened Y, direct Y])."""
    keep, args = _adapter_geo(cell, sigma)
    cubes = np.zeros(cell.n_atoms * len(cell.proj_l) * 6, dtype=np.int32)
    sums = np.zeros(4)
    code = adapter_lib().adapter_flatten_stats(*args, _ptr(cubes, _ip), _ptr(sums, _dp))
    return code, cubes.reshape(-1, 6), sums


def adapter_apply(cell, sigma, X):
    """(HX through the adapter on the GPU, HX of the reference integrator)."""
    keep, args = _adapter_geo(cell, sigma)
    X = _c64(X)
    hg, hr = np.zeros_like(X), np.zeros_like(X)
    rc = adapter_lib().adapter_apply_check(*args, X.shape[0], _ptr(X, _dp), _ptr(hg, _dp), _ptr(hr, _dp))
    if rc != 0:
        raise RuntimeError("adapter_apply_check failed")
    return hg, hr


def adapter_lobpcg(cell, sigma, X0, iter_max):
    """(ev of EigenLOBPCG_d_multi with the reference lambda, ev with the adapter's
    GpuOperator, the reference's iteration count)."""
    keep, args = _adapter_geo(cell, sigma)
    X0 = _c64(X0)
    er, eg = np.zeros(X0.shape[0]), np.zeros(X0.shape[0])
    it = C.c_int()
    rc = adapter_lib().adapter_lobpcg_check(*args, X0.shape[0], iter_max, _ptr(X0, _dp), _ptr(er, _dp),
                                            _ptr(eg, _dp), C.byref(it))
    if rc != 0:
        raise RuntimeError("adapter_lobpcg_check failed")
    return er, eg, it.value
