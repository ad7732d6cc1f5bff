"""Known-answer tests of the oracle's exact Euler Riemann solver and the
shock-bubble problem (CPU only).

Published reference values: E. F. Toro, Riemann Solvers and Numerical Methods for
Fluid Dynamics, Table 4.3 (exact star states of tests 1-5, gamma = 1.4, 5-6
significant digits)."""
import numpy as np
import pytest

from oracle import pyoracle as po

G = 1.4
TORO = [  # WL (rho, u, p), WR, p*, u*, rho*L, rho*R
    ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 0.30313, 0.92745, 0.42632, 0.26557),
    ((1.0, -2.0, 0.4), (1.0, 2.0, 0.4), 0.00189, 0.00000, 0.02185, 0.02185),
    ((1.0, 0.0, 1000.0), (1.0, 0.0, 0.01), 460.894, 19.5975, 0.57506, 5.99924),
    ((1.0, 0.0, 0.01), (1.0, 0.0, 100.0), 46.0950, -6.19633, 5.99242, 0.57511),
    ((5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.0950), 1691.64, 8.68975, 14.2823, 31.0426),
]


def _fk(p, r, pk):
    """Toro's pressure function and its derivative, numpy FP64."""
    a = np.sqrt(G * pk / r)
    if p <= pk:
        return 2 * a / (G - 1) * ((p / pk) ** ((G - 1) / (2 * G)) - 1)
    A, B = 2 / ((G + 1) * r), (G - 1) / (G + 1) * pk
    return (p - pk) * np.sqrt(A / (p + B))


def test_own_exp_log_pow_accuracy():
    rng = np.random.default_rng(0)
    L = po.lib()
    for x in np.concatenate([rng.uniform(1e-6, 1e6, 2000), rng.uniform(0.5, 2.0, 2000)]):
        assert abs(L.orc_log(x) - np.log(x)) <= 4e-16 * max(1.0, abs(np.log(x)))
    for y in rng.uniform(-40, 40, 4000):
        assert abs(L.orc_exp(y) - np.exp(y)) <= 2e-15 * np.exp(y)
    for x, a in zip(rng.uniform(1e-3, 1e3, 2000), rng.uniform(-3, 3, 2000)):
        ref = x ** a
        assert abs(L.orc_pow(x, a) - ref) <= 1e-14 * ref


@pytest.mark.parametrize("case", range(len(TORO)))
def test_toro_star_states(case):
    wl, wr, ps, us, rsl, rsr = TORO[case]
    out, it = po.euler_star(G, wl, wr, tol=1e-12)
    assert abs(out[0] - ps) <= 5e-5 * max(ps, 1e-3) + 6e-6
    assert abs(out[1] - us) <= 5e-5 * max(abs(us), 1.0)
    assert abs(out[2] - rsl) <= 5e-5 * rsl + 6e-6
    assert abs(out[3] - rsr) <= 5e-5 * rsr + 6e-6
    # pressure-function residual f_L(p*) + f_R(p*) + (uR - uL) = 0
    res = _fk(out[0], wl[0], wl[2]) + _fk(out[0], wr[0], wr[2]) + (wr[1] - wl[1])
    scale = abs(wl[1]) + abs(wr[1]) + np.sqrt(G * wl[2] / wl[0]) + np.sqrt(G * wr[2] / wr[0])
    assert abs(res) <= 1e-11 * scale
    assert 1 <= it <= 20


def test_rankine_hugoniot_of_shocks():
    # test 3: right-going shock into the right state
    wl, wr = TORO[2][0], TORO[2][1]
    out, _ = po.euler_star(G, wl, wr, tol=1e-12)
    ps, us, rsr = out[0], out[1], out[3]
    ar = np.sqrt(G * wr[2] / wr[0])
    sr = wr[1] + ar * np.sqrt((G + 1) / (2 * G) * ps / wr[2] + (G - 1) / (2 * G))
    mass_l, mass_r = rsr * (us - sr), wr[0] * (wr[1] - sr)
    mom_l, mom_r = rsr * us * (us - sr) + ps, wr[0] * wr[1] * (wr[1] - sr) + wr[2]
    assert abs(mass_l - mass_r) <= 1e-10 * abs(mass_r)
    assert abs(mom_l - mom_r) <= 1e-10 * abs(mom_r)


def _cons(w, v=0.0):
    r, u, p = w
    return np.array([r, r * u, r * v, p / (G - 1) + 0.5 * r * (u * u + v * v)])


def _flux(q):
    r, mu, mv, E = q
    u, v = mu / r, mv / r
    p = (G - 1) * (E - 0.5 * (mu * mu + mv * mv) / r)
    return np.array([mu, mu * u + p, mu * v, u * (E + p)])


@pytest.mark.parametrize("case", [0, 2, 3, 4])
def test_interface_consistency(case):
    wl, wr = TORO[case][0], TORO[case][1]
    ql, qr = _cons(wl, 0.3), _cons(wr, -0.2)
    w, s, am, ap, it = po.euler_interface(G, ql, qr)
    # the waves add up to the jump, the fluctuations to the flux difference
    assert np.allclose(w.sum(axis=0), qr - ql, rtol=0, atol=1e-12 * np.abs(qr - ql).max())
    df = _flux(qr) - _flux(ql)
    assert np.allclose(am + ap, df, rtol=0, atol=1e-12 * np.abs(df).max() + 1e-14)
    assert s[0] <= s[1] <= s[2]


def test_weak_waves_match_roe_linearisation():
    # for a small jump the exact fluctuations agree with the Roe split to O(jump^2)
    ql = _cons((1.0, 0.1, 1.0), 0.05)
    for eps in (1e-3, 1e-4):
        qr = ql + eps * np.array([1.0, 0.5, -0.3, 2.0])
        _, s, am, ap, _ = po.euler_interface(G, ql, qr)
        # Roe averages and the four-wave split (clawpack46_rpn2_euler4.f)
        rl, rr = np.sqrt(ql[0]), np.sqrt(qr[0])
        pl = (G - 1) * (ql[3] - 0.5 * (ql[1] ** 2 + ql[2] ** 2) / ql[0])
        pr = (G - 1) * (qr[3] - 0.5 * (qr[1] ** 2 + qr[2] ** 2) / qr[0])
        u = (ql[1] / rl + qr[1] / rr) / (rl + rr)
        v = (ql[2] / rl + qr[2] / rr) / (rl + rr)
        H = ((ql[3] + pl) / rl + (qr[3] + pr) / rr) / (rl + rr)
        a = np.sqrt((G - 1) * (H - 0.5 * (u * u + v * v)))
        d = qr - ql
        a3 = (G - 1) / a ** 2 * ((H - u * u - v * v) * d[0] + u * d[1] + v * d[2] - d[3])
        a2 = d[2] - v * d[0]
        a4 = (d[1] + (a - u) * d[0] - a * a3) / (2 * a)
        a1 = d[0] - a3 - a4
        w1 = a1 * np.array([1, u - a, v, H - u * a])
        amdq_roe = (u - a) * w1 if u - a < 0 else 0 * w1
        assert np.abs(am - amdq_roe).max() <= 50 * eps ** 2


def test_seed_at_solution_converges_in_one_step():
    wl, wr = TORO[0][0], TORO[0][1]
    out, it_pvrs = po.euler_star(G, wl, wr, tol=1e-10)
    _, it_seed = po.euler_star(G, wl, wr, seed=out[0], tol=1e-10)
    assert it_seed == 1 and it_pvrs > it_seed


def _shockbubble(**kw):
    d = dict(mx=8, my=8, mbc=2, meqn=4, maux=0, mwaves=3, mthlim=(4, 4, 4), rp=po.RP_EULER_EXACT,
             problem=po.PROB_SHOCKBUBBLE, mthbc=(0, 1, 3, 3), ax=0.0, bx=2.0, ay=0.0, by=1.0, mi=2, mj=1,
             x0=0.5, y0=0.5, r0=0.2, gamma=1.4, mach=1.22, rhob=0.138, newton_tol=1e-10,
             minlevel=2, maxlevel=3, subcycle=1, time_sync=1, refine_threshold=0.05, coarsen_threshold=0.01)
    d.update(kw)
    return po.OracleSim(po.make_config(**d))


def test_shockbubble_symmetry_and_conservation():
    s = _shockbubble()
    s.initialize()
    q0 = s.get_q()
    info = s.patch_info()
    m0 = s.mass()
    t, dt = 0.0, 0.004
    for _ in range(6):
        cfl = s.advance(t, dt)
        t += dt
        dt *= 0.8 / cfl
    q = s.get_q()
    assert np.isfinite(q).all()
    # mirror symmetry about y = 1/2: rho, m_x, E even, m_y odd
    lev, gx, gy = info[:, 0], info[:, 2], info[:, 3]
    key = {(l, x, y): k for k, (l, x, y) in enumerate(zip(lev, gx, gy))}
    nchk = 0
    scale = np.abs(q[:, :, 2:-2, 2:-2]).max(axis=(0, 2, 3))
    for k, (l, x, y) in enumerate(zip(lev, gx, gy)):
        j = key.get((l, x, (1 << l) - 1 - y))
        if j is None:
            continue
        a, b = q[k][:, 2:-2, 2:-2], q[j][:, 2:-2, 2:-2][:, ::-1, :]
        for m, sg in ((0, 1), (1, 1), (2, -1), (3, 1)):
            assert np.allclose(a[m], sg * b[m], rtol=0, atol=1e-12 * scale[m])
        nchk += 1
    assert nchk == len(lev)
    # inflow adds mass through the left boundary: bounded, positive change
    m1 = s.mass()
    assert m1[0] > m0[0]
    hist = po.newton_hist(reset=True)
    # bin 0: interfaces without a pressure / normal-velocity jump (no Newton step)
    assert hist[0] > 0 and hist[1:].sum() > 0
