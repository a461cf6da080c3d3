"""An independent numpy restatement of the fast Ewald method, for cross-checking
the C++ oracle on small inputs (TEST INFRASTRUCTURE).

It follows the same equations as the reference (fft/ewald_fft_3d_real.f90,
fft/ewald_fft_3d_fourier.f90, nfft/nfft.f90) but is written independently:
brute-force image sums in real space, np.add.at spreading and numpy's pocketfft
in place of FFTW."""

import math

import numpy as np


def real_space(pos, q, lat_rows, alpha, r_cut):
    lat = np.asarray(lat_rows)
    rec = np.linalg.inv(lat).T  # rows b_i with b_i . a_j = delta_ij
    n_img = [int(math.ceil(r_cut * np.linalg.norm(rec[d]))) + 1 for d in range(3)]
    shifts = np.array([[i, j, k] for i in range(-n_img[0], n_img[0] + 1)
                       for j in range(-n_img[1], n_img[1] + 1)
                       for k in range(-n_img[2], n_img[2] + 1)], dtype=float) @ lat
    N = len(q)
    pot = np.zeros(N)
    force = np.zeros((N, 3))
    for i in range(N):
        d = pos[i][None, None, :] - pos[None, :, :] + shifts[:, None, :]  # (S, N, 3)
        r2 = np.sum(d * d, axis=-1)
        mask = r2 <= r_cut * r_cut
        zero = np.all(np.abs(shifts) < 1e-300, axis=1)[:, None] & (np.arange(N)[None, :] == i)
        mask &= ~zero
        r = np.sqrt(np.where(mask, r2, 1.0))
        from scipy.special import erfc
        ec = erfc(alpha * r)
        pot[i] = np.sum(np.where(mask, q[None, :] * ec / r, 0.0))
        ff = q[i] * q[None, :] * (2 * alpha / math.sqrt(math.pi) * np.exp(-alpha * alpha * r * r) + ec / r) / (r * r)
        force[i] = np.sum(np.where(mask[..., None], ff[..., None] * d, 0.0), axis=(0, 1))
    return pot, force


def _mode(a, M):
    return a - M if a >= M // 2 else a


def fourier(pos, q, lat_rows, alpha, M, m):
    lat = np.asarray(lat_rows)
    rec = np.linalg.inv(lat).T
    V = abs(np.linalg.det(lat))
    t = pos @ rec.T  # fractional coordinates
    n = [2 * Md for Md in M]
    b = (4.0 / 3.0) * (m / math.pi)
    pref = 1.0 / math.sqrt(math.pi * b)
    off = np.arange(-m, m + 1)

    def weights(td, nd):
        w = td - np.floor(td)
        s = w * nd
        lo = np.floor(s).astype(int)
        frac = s - lo
        lo = np.where(lo >= nd, lo - nd, lo)
        wt = pref * np.exp(-(frac[:, None] - off[None, :]) ** 2 / b)
        idx = (lo[:, None] + off[None, :]) % nd
        return idx, wt

    idx = []
    wts = []
    for d in range(3):
        i_, w_ = weights(t[:, d], n[d])
        idx.append(i_)
        wts.append(w_)
    grid = np.zeros(n)
    for j in range(len(q)):
        W = q[j] * wts[0][j][:, None, None] * wts[1][j][None, :, None] * wts[2][j][None, None, :]
        np.add.at(grid, np.ix_(idx[0][j], idx[1][j], idx[2][j]), W)
    Gp = np.fft.ifftn(grid) * grid.size  # sign +1, unnormalised
    k_axes = [np.array([_mode(a, M[d]) for a in range(M[d])]) for d in range(3)]
    fac = [np.exp(b * (math.pi * k_axes[d] / n[d]) ** 2) for d in range(3)]
    shat = Gp[np.ix_(k_axes[0] % n[0], k_axes[1] % n[1], k_axes[2] % n[2])]
    corr = fac[0][:, None, None] * fac[1][None, :, None] * fac[2][None, None, :]
    shat = shat * corr
    K = np.stack(np.meshgrid(*k_axes, indexing="ij"), -1).astype(float)
    kv = 2 * math.pi * K @ rec  # Cartesian wave vectors
    k2 = np.sum(kv * kv, -1)
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.where(k2 < 1e-24, 0.0, 4 * math.pi / V * np.exp(-k2 / (4 * alpha * alpha)) / k2)
    coef = w * shat

    def forward(fh):
        fine = np.zeros(n, dtype=complex)
        fine[np.ix_(k_axes[0] % n[0], k_axes[1] % n[1], k_axes[2] % n[2])] = fh * corr
        f = np.fft.fftn(fine)
        out = np.zeros(len(q), dtype=complex)
        for j in range(len(q)):
            W = wts[0][j][:, None, None] * wts[1][j][None, :, None] * wts[2][j][None, None, :]
            out[j] = np.sum(W * f[np.ix_(idx[0][j], idx[1][j], idx[2][j])])
        return out

    pot = forward(coef).real
    force = np.zeros((len(q), 3))
    for c in range(3):
        force[:, c] = q * forward(1j * kv[..., c] * coef).real
    return pot, force


def potential_force(pos, q, lat_rows, alpha, r_cut, M, m):
    sp, sf = real_space(pos, q, lat_rows, alpha, r_cut)
    lp, lf = fourier(pos, q, lat_rows, alpha, M, m)
    return sp + lp - 2 * alpha / math.sqrt(math.pi) * q, sf + lf
