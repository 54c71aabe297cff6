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
        lib.ref_lobpcg_d_multi.argtypes = [C.POINTER(HamDescC), C.c_int, C.c_int, _dp, _dp, _dp,
                                           C.c_int, C.c_int, _ip]
        lib.ref_grid_for_sphere.argtypes = [C.c_double] * 7 + [_ip]
        lib.ref_ylm_cube.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp]
        lib.ref_hamiltonian_kpoint_apply.argtypes = [C.POINTER(HamDescC), C.c_double, C.c_double,
                                                     C.c_double, C.c_double, C.c_int, _dp, _dp]
        lib.ref_lobpcg_z_multi.argtypes = [C.POINTER(HamDescC), C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.c_int, C.c_int, _dp, _dp, C.c_int, _ip]
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


def hamiltonian_kpoint_apply(cell, g, X, impl="port"):
    """Complex k-point H (V + nonlocal with Bloch phases + 8th-order k-point kinetic)
    on {re, im} states X (ns, 2N); g = Bloch vector in bohr^-1."""
    X = _c64(X)
    HX = np.zeros_like(X)
    desc = HamDesc(cell, 8)
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
