"""FP64 reference of the force adjoint (vector-Jacobian product), numpy.

Test infrastructure: the checker for the library's adjoint kernels, itself
checked against central finite differences of the oracle's forces.  Nothing in
the library imports it.

The force is the one of an RBL + RBE step with fixed lists and fixed k-samples
(LJCutCoulKspace::ComputeLJRBL and KSpaceCalculator::ComputeRBE,
lj_cut_coul_kspace.cpp:494-573, kspace_calculator.cpp:532-588):

    F_i = P_i - (1/N) sum_j P_j + K_i
    P_i = sum_{(i,j,s) in RBL lists} s f(r_ij^2) d_ij,   d_ij = r_j - r_i
    f   = LJ  -24 eps_ij (2 u^2 - u) / r^2,  u = sigma_ij^6 / r^6
        + Coulomb  q_i q_j h(r),  h = -qqr2e (erfc(b r)/r^2 + 2b e^{-a r^2}/(sqrt(pi) r)) / r,
          b = sqrt(a)                                     (lj_op.hip.cu:40-73,
                                                     lj_cut_coul_kspace_op.hip.cu:134-194)
    K_i = q_i sum_k c_k (cos(k.r_i) Im rho_k - sin(k.r_i) Re rho_k) k,
          c_k = -4 pi qqr2e S(a) / (P V k^2),  rho_k = sum_j q_j e^{i k.r_j}
                                                     (kspace_calculator_op.hip.cu:98-125)
    eps_ij = sqrt(eps_ti eps_tj), sigma_ij = (sigma_ti + sigma_tj) / 2.

Given g = dL/dF it returns dL/d(eps_t), dL/d(sigma_t), dL/dq_i, dL/dalpha and
dL/dr_i.  With g' = g - mean(g) (the mean removal is linear), a pair
contributes s (df/dtheta)(g'_i . d) to the parameters and
c = s (f g'_i + 2 f'(g'_i . d) d), f' = df/d(r^2), to dL/dr_j (and -c to dL/dr_i).
The k-space part uses a_k = sum_i q_i (g_i.k) cos(k.r_i) and
b_k = sum_i q_i (g_i.k) sin(k.r_i):
    dL/dq_m = sum_k c_k [(g_m.k)(cos Im rho - sin Re rho) + a_k sin - b_k cos]
    dL/dr_m = q_m sum_k c_k k [-(g_m.k)(sin Im rho + cos Re rho) + a_k cos + b_k sin]
    dL/dalpha (k-space) = (S'(a)/S(a)) sum_m g_m . K_m.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erfc

RBX_EPSILON = 1e-4


def rbl_pairs(cc, core, sc, shell, freq):
    """(i, j, scale, is_core) arrays of the RBL lists (rows of capacity cap)."""
    n = len(cc)
    ii, jj, ss, kk = [], [], [], []
    for i in range(n):
        js = core[i, :cc[i]]
        ii.append(np.full(len(js), i))
        jj.append(js)
        ss.append(np.ones(len(js)))
        kk.append(np.ones(len(js), bool))
        js = shell[i, :sc[i]]
        ii.append(np.full(len(js), i))
        jj.append(js)
        ss.append(np.full(len(js), float(freq)))
        kk.append(np.zeros(len(js), bool))
    return (np.concatenate(ii).astype(int), np.concatenate(jj).astype(int), np.concatenate(ss),
            np.concatenate(kk))


def _min_image(d, L):
    return d - L * np.rint(d / L)


def pair_terms(pos, L, typ, sigma, eps, q, alpha, qqr2e, i, j, is_core, r_core, cut_off):
    """f, df/d(r^2) and the parameter partials of every listed pair (window applied)."""
    d = _min_image(pos[j] - pos[i], L)
    r2 = (d ** 2).sum(1)
    rs2, rc2 = r_core ** 2, cut_off ** 2
    active = np.where(is_core, (r2 < rs2) & (r2 > RBX_EPSILON), (r2 < rc2) & (r2 > rs2))
    ti, tj = typ[i], typ[j]
    e = np.sqrt(eps[ti] * eps[tj])
    sg = 0.5 * (sigma[ti] + sigma[tj])
    ui = 1.0 / r2
    s6 = sg ** 6
    u = s6 * ui ** 3                      # sigma^6 / r^6
    f_lj = -24 * e * (2 * u * u - u) * ui
    # df/d(r^2) of the LJ term: 24 eps (14 s12 u^8 - 4 s6 u^5) in u = 1/r^2
    fp_lj = 24 * e * (14 * s6 * s6 * ui ** 8 - 4 * s6 * ui ** 5)
    df_de = f_lj / e
    df_ds = -144 * e * (4 * u * u - u) * ui / sg
    r = np.sqrt(r2)
    b = math.sqrt(alpha)
    ex = np.exp(-alpha * r2)
    h = -qqr2e * (erfc(b * r) * ui + 2 * b * ex / (math.sqrt(math.pi) * r)) / r
    dh_dr = qqr2e * (3 * erfc(b * r) / r ** 4
                     + 2 * b / math.sqrt(math.pi) * ex * (3 / r ** 3 + 2 * alpha / r))
    dh_da = 2 * qqr2e * b * ex / math.sqrt(math.pi)
    qq = q[i] * q[j]
    f = np.where(active, f_lj + qq * h, 0.0)
    fp = np.where(active, fp_lj + qq * dh_dr / (2 * r), 0.0)
    z = lambda a: np.where(active, a, 0.0)  # noqa: E731
    return d, f, fp, z(df_de), z(df_ds), z(h), z(qq * dh_da)


def gauss_sum_and_derivative(L, alpha):
    """S(alpha) = prod_d H_d - 1 (kspace_calculator.cpp:68-78) and dS/dalpha."""
    H, dH = [], []
    m = np.arange(-10, 11)
    for Ld in L:
        w = np.exp(-alpha * Ld * Ld * m * m)
        pre = math.sqrt(alpha * Ld * Ld / math.pi)
        H.append(pre * w.sum())
        dH.append(pre * w.sum() / (2 * alpha) - pre * (Ld * Ld * m * m * w).sum())
    S = H[0] * H[1] * H[2] - 1
    dS = dH[0] * H[1] * H[2] + H[0] * dH[1] * H[2] + H[0] * H[1] * dH[2]
    return S, dS


def force_vjp(pos, L, typ, sigma, eps, q, alpha, qqr2e, r_core, cut_off, freq, lists, m, g):
    """(d_eps[ntypes], d_sigma[ntypes], d_q[n], d_alpha, d_r[n,3]) for upstream g = dL/dF."""
    n = len(pos)
    nt = len(sigma)
    i, j, s, is_core = lists
    gp = g - g.mean(0)
    d, f, fp, df_de, df_ds, h, dfq_da = pair_terms(pos, L, typ, sigma, eps, q, alpha, qqr2e,
                                                   i, j, is_core, r_core, cut_off)
    gd = (gp[i] * d).sum(1)
    w = s * gd
    d_eps = np.zeros(nt)
    d_sig = np.zeros(nt)
    e_ij = np.sqrt(eps[typ[i]] * eps[typ[j]])
    for end in (typ[i], typ[j]):  # each end carries half of d(eps_ij)/d(eps_t) and d(sigma_ij)
        np.add.at(d_eps, end, w * df_de * e_ij / (2 * eps[end]))
        np.add.at(d_sig, end, w * df_ds * 0.5)
    d_q = np.zeros(n)
    np.add.at(d_q, i, w * h * q[j])
    np.add.at(d_q, j, w * h * q[i])
    d_alpha = float((w * dfq_da).sum())
    c = s[:, None] * (f[:, None] * gp[i] + 2 * fp[:, None] * gd[:, None] * d)
    d_r = np.zeros((n, 3))
    np.add.at(d_r, j, c)
    np.add.at(d_r, i, -c)
    # k-space
    V = float(np.prod(L))
    P = len(m[0])
    k = np.stack([2 * math.pi * np.asarray(m[a]) / L[a] for a in range(3)], 1)  # [P, 3]
    k2 = (k ** 2).sum(1)
    S, dS = gauss_sum_and_derivative(L, alpha)
    ck = -4 * math.pi * qqr2e * S / (P * V * k2)
    th = pos @ k.T                                                             # [n, P]
    cs, sn = np.cos(th), np.sin(th)
    re, im = q @ cs, q @ sn
    gk = g @ k.T                                                               # g_i . k
    a_k = (q[:, None] * gk * cs).sum(0)
    b_k = (q[:, None] * gk * sn).sum(0)
    d_q += ((gk * (cs * im - sn * re) + a_k * sn - b_k * cs) * ck).sum(1)
    coef = ck * (-gk * (sn * im + cs * re) + a_k * cs + b_k * sn)             # [n, P]
    d_r += q[:, None] * (coef @ k)
    fk = q[:, None] * ((ck * (cs * im - sn * re)) @ k)                         # K_i
    d_alpha += dS / S * float((g * fk).sum())
    return d_eps, d_sig, d_q, d_alpha, d_r
