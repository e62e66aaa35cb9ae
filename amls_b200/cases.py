"""Input pencils: the reference's closed-form cases and seeded hex-elasticity pencils.

The closed-form generators and spectra restate ``src/io/case_generator.cpp``
(path graph :15-54, 2-D grid :56-93, 3-D grid :95-146) so that the same known
answers the reference's tests use (``tests/unit/test_io.cpp:31-79``,
``tests/unit/test_amls.cpp:110-151``) can be checked here.

The hex-elasticity pencils are the synthetic FEM inputs of the benchmark
configurations: a box of ``ex x ey x ez`` cubic elements of side ``h``,
trilinear 8-node (2x2x2 Gauss) or triquadratic 27-node (3x3x3 Gauss),
3 displacement DOFs per node, isotropic linear elasticity (nu = 0.3) and
consistent mass, all nodes on the face x = 0 clamped.  Element moduli and
densities are scaled per element: E_e = u_e ~ U[0.5, 1.5], rho_e = v_e ~
U[0.8, 1.2], drawn from numpy's PCG64 with the given seed (u for all
elements first, then v, element-major).  Because every element is the same
cube, K = sum_e E_e Kbar and M = sum_e rho_e Mbar with one reference element
pair (Kbar, Mbar); the element data is kept on the returned pencil so that
eigenvalue sensitivities can be formed from it.

All matrices are returned as CSR with int64 row pointers, int32 column
indices (sorted within each row) and float64 values.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.sparse as sp


@dataclasses.dataclass
class Pencil:
    """A symmetric-definite pencil (K, M) in CSR, plus optional FEM data."""

    K: sp.csr_matrix
    M: sp.csr_matrix
    # element data (hex pencils only)
    dofmap: np.ndarray | None = None   # (nelem, ndof_e) int64, -1 = clamped
    Kbar: np.ndarray | None = None     # (ndof_e, ndof_e) element stiffness, E = 1
    Mbar: np.ndarray | None = None     # (ndof_e, ndof_e) element mass, rho = 1
    E: np.ndarray | None = None        # (nelem,) element moduli
    rho: np.ndarray | None = None      # (nelem,) element densities
    name: str = ""
    # mesh geometry (hex pencils only): node coordinates, element node ids
    coords: np.ndarray | None = None   # (nnodes, 3)
    enodes: np.ndarray | None = None   # (nelem, (order+1)^3) int64
    order: int = 0
    nu: float = 0.3

    @property
    def n(self) -> int:
        return self.K.shape[0]


def _csr(A) -> sp.csr_matrix:
    A = sp.csr_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    A.indptr = A.indptr.astype(np.int64)
    A.indices = A.indices.astype(np.int32)
    A.data = A.data.astype(np.float64)
    return A


# --------------------------------------------------------------------------
# closed-form cases (src/io/case_generator.cpp)
# --------------------------------------------------------------------------

def path_graph(n: int, consistent_mass: bool = False) -> Pencil:
    """Path Laplacian K = tridiag(-1, 2, -1); M = I or tridiag(1/6, 2/3, 1/6)
    (case_generator.cpp:15-40)."""
    i = np.arange(n)
    K = sp.diags([-np.ones(n - 1), 2.0 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1])
    if consistent_mass:
        M = sp.diags([np.full(n - 1, 1.0 / 6.0), np.full(n, 2.0 / 3.0),
                      np.full(n - 1, 1.0 / 6.0)], [-1, 0, 1])
    else:
        M = sp.identity(n)
    del i
    return Pencil(_csr(K), _csr(M), name=f"path:{n}")


def path_graph_spectrum(n: int, consistent_mass: bool = False) -> np.ndarray:
    """Ascending exact spectrum of :func:`path_graph` (case_generator.cpp:42-54)."""
    th = math.pi * np.arange(1, n + 1) / (n + 1)
    if consistent_mass:
        w = 6.0 * (1.0 - np.cos(th)) / (2.0 + np.cos(th))
    else:
        w = 2.0 - 2.0 * np.cos(th)
    return np.sort(w)


def grid_graph_2d(nx: int, ny: int) -> Pencil:
    """5-point Laplacian on nx x ny, vertex id = j*nx + i, M = I
    (case_generator.cpp:56-77)."""
    Tx = sp.diags([-np.ones(nx - 1), 2.0 * np.ones(nx), -np.ones(nx - 1)], [-1, 0, 1])
    Ty = sp.diags([-np.ones(ny - 1), 2.0 * np.ones(ny), -np.ones(ny - 1)], [-1, 0, 1])
    K = sp.kron(sp.identity(ny), Tx) + sp.kron(Ty, sp.identity(nx))
    return Pencil(_csr(K), _csr(sp.identity(nx * ny)), name=f"grid:{nx},{ny}")


def grid_graph_2d_spectrum(nx: int, ny: int) -> np.ndarray:
    """case_generator.cpp:79-93."""
    tx = 2.0 - 2.0 * np.cos(math.pi * np.arange(1, nx + 1) / (nx + 1))
    ty = 2.0 - 2.0 * np.cos(math.pi * np.arange(1, ny + 1) / (ny + 1))
    return np.sort((ty[:, None] + tx[None, :]).ravel())


def grid_graph_3d(nx: int, ny: int, nz: int) -> Pencil:
    """7-point Laplacian, vertex id = (k*ny + j)*nx + i, M = I
    (case_generator.cpp:95-122)."""
    def T(m):
        return sp.diags([-np.ones(m - 1), 2.0 * np.ones(m), -np.ones(m - 1)], [-1, 0, 1])
    Ix, Iy, Iz = sp.identity(nx), sp.identity(ny), sp.identity(nz)
    K = (sp.kron(Iz, sp.kron(Iy, T(nx))) + sp.kron(Iz, sp.kron(T(ny), Ix))
         + sp.kron(T(nz), sp.kron(Iy, Ix)))
    return Pencil(_csr(K), _csr(sp.identity(nx * ny * nz)), name=f"grid3d:{nx}")


def grid_graph_3d_spectrum(nx: int, ny: int, nz: int) -> np.ndarray:
    """case_generator.cpp:124-146."""
    def ax(m):
        return 2.0 - 2.0 * np.cos(math.pi * np.arange(1, m + 1) / (m + 1))
    w = ax(nz)[:, None, None] + ax(ny)[None, :, None] + ax(nx)[None, None, :]
    return np.sort(w.ravel())


# --------------------------------------------------------------------------
# hex elasticity pencils
# --------------------------------------------------------------------------

def _lagrange_1d(order: int):
    """Nodes, values and derivatives of the 1-D Lagrange basis on [-1, 1]."""
    nodes = np.linspace(-1.0, 1.0, order + 1)

    def basis(x):
        v = np.ones(order + 1)
        d = np.zeros(order + 1)
        for a in range(order + 1):
            for b in range(order + 1):
                if b == a:
                    continue
                v[a] *= (x - nodes[b]) / (nodes[a] - nodes[b])
            # derivative by the product rule
            s = 0.0
            for c in range(order + 1):
                if c == a:
                    continue
                t = 1.0 / (nodes[a] - nodes[c])
                for b in range(order + 1):
                    if b == a or b == c:
                        continue
                    t *= (x - nodes[b]) / (nodes[a] - nodes[b])
                s += t
            d[a] = s
        return v, d

    return nodes, basis


def hex_element_matrices(order: int, h: float, nu: float = 0.3):
    """Reference element stiffness (E = 1) and consistent mass (rho = 1) of a
    cubic hex element of side h.  DOF index = 3*local_node + component, local
    node = a + (p+1)*(b + (p+1)*c) for 1-D node indices (a, b, c)."""
    p = order
    nn1 = p + 1
    nn = nn1 ** 3
    gx, gw = np.polynomial.legendre.leggauss(p + 1)
    _, basis = _lagrange_1d(p)
    lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = 1.0 / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2.0 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    jac = h / 2.0
    detJ = jac ** 3
    Ke = np.zeros((3 * nn, 3 * nn))
    Me = np.zeros((3 * nn, 3 * nn))
    for ix, xi in enumerate(gx):
        vx, dx = basis(xi)
        for iy, eta in enumerate(gx):
            vy, dy = basis(eta)
            for iz, zeta in enumerate(gx):
                vz, dz = basis(zeta)
                w = gw[ix] * gw[iy] * gw[iz] * detJ
                N = np.einsum("c,b,a->cba", vz, vy, vx).ravel()
                dNx = np.einsum("c,b,a->cba", vz, vy, dx).ravel() / jac
                dNy = np.einsum("c,b,a->cba", vz, dy, vx).ravel() / jac
                dNz = np.einsum("c,b,a->cba", dz, vy, vx).ravel() / jac
                B = np.zeros((6, 3 * nn))
                B[0, 0::3] = dNx
                B[1, 1::3] = dNy
                B[2, 2::3] = dNz
                B[3, 0::3] = dNy
                B[3, 1::3] = dNx
                B[4, 1::3] = dNz
                B[4, 2::3] = dNy
                B[5, 0::3] = dNz
                B[5, 2::3] = dNx
                Ke += w * (B.T @ D @ B)
                NN = np.outer(N, N) * w
                for c in range(3):
                    Me[c::3, c::3] += NN
    Ke = 0.5 * (Ke + Ke.T)
    Me = 0.5 * (Me + Me.T)
    return Ke, Me


def hex_pencil(ex: int, ey: int, ez: int, order: int, seed: int = 0,
               h: float | None = None, nu: float = 0.3) -> Pencil:
    """Seeded hex-elasticity pencil on an ex x ey x ez box, face x = 0 clamped.

    order 1 = 8-node trilinear, order 2 = 27-node triquadratic.  The element
    side defaults to 1/max(ex, ey, ez) (the unit cube for ex = ey = ez).
    """
    if order not in (1, 2):
        raise ValueError("order must be 1 (8-node) or 2 (27-node)")
    p = order
    if h is None:
        h = 1.0 / max(ex, ey, ez)
    nx, ny, nz = p * ex + 1, p * ey + 1, p * ez + 1
    gnode = np.arange(nx * ny * nz).reshape(nz, ny, nx)  # id = i + nx*(j + ny*k)
    free = np.ones((nz, ny, nx), dtype=bool)
    free[:, :, 0] = False
    fidx = -np.ones(nx * ny * nz, dtype=np.int64)
    fidx[gnode[free].ravel()] = np.arange(int(free.sum()))
    n = 3 * int(free.sum())

    nn1 = p + 1
    la, lb, lc = np.meshgrid(np.arange(nn1), np.arange(nn1), np.arange(nn1), indexing="ij")
    # local node = a + nn1*(b + nn1*c)  -> arrays indexed by that order
    loc_a = np.zeros(nn1 ** 3, dtype=np.int64)
    loc_b = np.zeros_like(loc_a)
    loc_c = np.zeros_like(loc_a)
    for c in range(nn1):
        for b in range(nn1):
            for a in range(nn1):
                ln = a + nn1 * (b + nn1 * c)
                loc_a[ln], loc_b[ln], loc_c[ln] = a, b, c
    del la, lb, lc
    eX, eY, eZ = np.meshgrid(np.arange(ex), np.arange(ey), np.arange(ez), indexing="ij")
    # element index = ex_i + ex*(ey_j + ey*ez_k)
    eX = eX.transpose(2, 1, 0).ravel()
    eY = eY.transpose(2, 1, 0).ravel()
    eZ = eZ.transpose(2, 1, 0).ravel()
    gi = p * eX[:, None] + loc_a[None, :]
    gj = p * eY[:, None] + loc_b[None, :]
    gk = p * eZ[:, None] + loc_c[None, :]
    enodes = gi + nx * (gj + ny * gk)                      # (nelem, nn)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    coords = np.zeros((nx * ny * nz, 3))
    gid = (ii + nx * (jj + ny * kk)).ravel()
    coords[gid, 0] = ii.ravel() * (h / p)
    coords[gid, 1] = jj.ravel() * (h / p)
    coords[gid, 2] = kk.ravel() * (h / p)
    fn = fidx[enodes]                                       # -1 where clamped
    dofmap = np.where(fn[:, :, None] >= 0, 3 * fn[:, :, None] + np.arange(3)[None, None, :], -1)
    dofmap = dofmap.reshape(fn.shape[0], -1)                # DOF = 3*local_node + comp

    nelem = ex * ey * ez
    rng = np.random.Generator(np.random.PCG64(seed))
    E = rng.uniform(0.5, 1.5, nelem)
    rho = rng.uniform(0.8, 1.2, nelem)
    Kbar, Mbar = hex_element_matrices(order, h, nu)

    K = _assemble(dofmap, Kbar, E, n)
    M = _assemble(dofmap, Mbar, rho, n)
    name = f"hex{8 if order == 1 else 27}:{ex}x{ey}x{ez}:seed{seed}"
    return Pencil(K, M, dofmap=dofmap, Kbar=Kbar, Mbar=Mbar, E=E, rho=rho, name=name, coords=coords,
                  enodes=enodes.astype(np.int64), order=order, nu=nu)


def _assemble(dofmap: np.ndarray, Ae: np.ndarray, scale: np.ndarray, n: int) -> sp.csr_matrix:
    nd = dofmap.shape[1]
    rows = np.broadcast_to(dofmap[:, :, None], (dofmap.shape[0], nd, nd))
    cols = np.broadcast_to(dofmap[:, None, :], (dofmap.shape[0], nd, nd))
    keep = (rows >= 0) & (cols >= 0)
    vals = scale[:, None, None] * Ae[None, :, :]
    A = sp.coo_matrix((vals[keep], (rows[keep], cols[keep])), shape=(n, n))
    A = _csr(A)
    # exact symmetry (assembly sums are order-dependent in the last bit)
    At = _csr(A.T)
    A.data = 0.5 * (A.data + At.data)
    return A


# --------------------------------------------------------------------------
# benchmark configurations
# --------------------------------------------------------------------------

def config_pencil(name: str, seed: int = 0) -> Pencil:
    """The named synthetic pencils: C1 8-node 12^3 (6,084 DOF), C2 27-node 7^3
    (9,450), C4 27-node 10^3 (26,460), C5 27-node 14^3 (70,644)."""
    table = {"C1": (12, 1), "C2": (7, 2), "C4": (10, 2), "C5": (14, 2)}
    e, order = table[name]
    return hex_pencil(e, e, e, order, seed=seed)


def batch_shapes(count: int = 256, seed: int = 0, lo: int = 4, hi: int = 12):
    """Box shapes (a, b, c) ~ U{lo..hi} for the uneven pencil batch."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [tuple(int(v) for v in rng.integers(lo, hi + 1, size=3)) for _ in range(count)]


def batch_pencils(count: int = 256, seed: int = 0, lo: int = 4, hi: int = 12) -> list[Pencil]:
    """The uneven batch: 8-node hex elasticity boxes of a x b x c elements
    (a, b, c ~ U{lo..hi}), face x = 0 clamped, the E / rho perturbation law
    of hex_pencil with a seed per pencil (seed * 1000003 + b + 1)."""
    return [hex_pencil(a, b_, c, 1, seed=seed * 1000003 + q + 1)
            for q, (a, b_, c) in enumerate(batch_shapes(count, seed, lo, hi))]
