"""The boundary-transfer form of vort2flux! (ibpm.jl_b200/csrc/bt.cu), restated
in numpy with the kernels' index conventions and checked against the oracle's
vort2flux (src/fluid-operators/curl.jl:133-165) on the CPU:

* every level's interior part Δ⁻¹Γ_ℓ from one x-pass and one y-pass;
* the line samples of the y-pass output (rows at ny/4, 3ny/4 by an inverse
  x-transform; columns at nx/4, 3nx/4 by the period-8 weights 2 sin(πk/4),
  2 sin(3πk/4));
* the edge chain e_ℓ = get_bc!(samples of ℓ+1) + R e_{ℓ+1}, R built column
  by column from unit edge sources;
* the x-spectrum of apply_bc!(e_ℓ) in closed form, one y-pass, and one x-pass
  of the sum.
The identity is exact; the check is to rounding."""
import numpy as np
import pytest
import scipy.fft as sfft

from oracle import ibpm_ref as R


def dst1(x, axis):
    return sfft.dst(x, type=1, axis=axis)          # Y_k = 2 Σ f_m sin(π m k / N)


def edge_point(k, n1, n2):
    if k < n1:
        return k, 0
    if k < 2 * n1:
        return k - n1, n2 - 1
    if k < 2 * n1 + n2:
        return 0, k - 2 * n1
    return n1 - 1, k - 2 * n1 - n2


def bc_used(psi, g):
    """The entries of get_bc!(psi) that apply_bc! adds (bottom, top, left, right)."""
    bc = R.get_bc(psi, g)
    nx, ny = g.nx, g.ny
    return np.concatenate([bc[g.BOT + 1:g.BOT + nx], bc[g.TOP + 1:g.TOP + nx],
                           bc[g.LEFT + 1:g.LEFT + ny], bc[g.RIGHT + 1:g.RIGHT + ny]])


def samples(Y, g):
    nx, ny, n1 = g.nx, g.ny, g.nx - 1
    o0, o1 = nx // 4 - 1, 3 * nx // 4 - 1
    rowB = dst1(Y[:, ny // 4 - 1], 0)[o0:o1 + 1]
    rowT = dst1(Y[:, 3 * ny // 4 - 1], 0)[o0:o1 + 1]
    s2 = np.sqrt(2.0)
    k = (np.arange(n1) + 1) & 7
    wl = np.array([0, s2, 2, s2, 0, -s2, -2, -s2])[k]
    wr = np.array([0, s2, -2, s2, 0, -s2, 2, -s2])[k]
    rows = Y[:, ny // 4 - 1:3 * ny // 4]
    return rowB, rowT, wl @ rows, wr @ rows


def edge_from_samples(smp, g):
    def seg(s, n):
        v = np.arange(1, n)
        return np.where(v % 2 == 0, s[v // 2], 0.5 * (s[(v + 1) // 2] + s[(v - 1) // 2]))
    rowB, rowT, colL, colR = smp
    return np.concatenate([seg(rowB, g.nx), seg(rowT, g.nx), seg(colL, g.ny), seg(colR, g.ny)])


def vort2flux_bt(G, g):
    nx, ny, mg = g.nx, g.ny, G.shape[0]
    n1, n2 = nx - 1, ny - 1
    Lam, scale = R.lap_eigs(g), R.lap_inv_scale(g)
    for lev in range(1, mg):
        R.coarsify(G[lev], G[lev - 1], g)
    nE = 2 * n1 + 2 * n2
    Rm = np.zeros((nE, nE))
    for k in range(nE):
        f = np.zeros((n1, n2))
        f[edge_point(k, n1, n2)] = 1.0
        Rm[:, k] = bc_used(R.dst_inv(f, Lam, scale), g)
    Y = dst1(dst1(dst1(G, 1), 2) / Lam * scale, 2)
    e = np.zeros((mg, nE))
    for lev in range(mg - 2, -1, -1):
        e[lev] = edge_from_samples(samples(Y[lev + 1], g), g) + (Rm @ e[lev + 1] if lev < mg - 2 else 0.0)
    sinpix = lambda t: np.sin(np.pi * (t % (2 * nx)) / nx)
    k = np.arange(1, nx)
    S = 2 * sinpix(np.outer(k, k))                  # S[i-1, k-1] = 2 sin(π i k / nx)
    for lev in range(mg - 1):
        eB, eT = e[lev, :n1], e[lev, n1:2 * n1]
        eL, eR = e[lev, 2 * n1:2 * n1 + n2], e[lev, 2 * n1 + n2:]
        X = np.outer(2 * sinpix(k), eL) + np.outer(2 * sinpix(k * (nx - 1)), eR)
        X[:, 0] += S.T @ eB
        X[:, n2 - 1] += S.T @ eT
        Y[lev] += dst1(dst1(X, 1) / Lam * scale, 1)
    return dst1(Y, 1)


@pytest.mark.parametrize("bnd,nx,mg", [((-2.0, 2.0, -2.0, 2.0), 32, 4), ((-2.0, 2.0, -1.0, 1.0), 64, 3),
                                       ((-1.0, 3.0, -2.0, 2.0), 40, 2)])
def test_boundary_transfer_equals_vort2flux(bnd, nx, mg):
    g = R.make_grid((bnd[1] - bnd[0]) / nx, bnd, mg)
    rng = np.random.default_rng(nx + mg)
    G = rng.standard_normal((mg, g.nx - 1, g.ny - 1))
    psi_ref, _, _ = R.vort2flux(G.copy(), R.lap_eigs(g), g)
    psi = vort2flux_bt(G.copy(), g)
    assert np.max(np.abs(psi - psi_ref)) / np.max(np.abs(psi_ref)) < 1e-13
