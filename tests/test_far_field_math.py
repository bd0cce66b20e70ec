"""The algebra of the per-facet forward's FP32 mid field (kernels_facet.cuh,
pair_far_f32<RULE_MID>, atanh_q_any), restated in numpy and checked on the
CPU: the Gauss-Green form of the facet's 1/r integral, its regrouping around
the mean vertex-distance sum, and the half-argument steps for
atanh(e)/e - 1.  The GPU parity tests check the kernels themselves against
the oracle; these check that the formulas they evaluate are exact, and
that the FP32 steps do not cancel.  CPU only."""
import numpy as np
import pytest


def _frame(a, b, c):
    L0 = np.linalg.norm(b - a)
    xh = (b - a) / L0
    n = np.cross(b - a, c - a)
    zh = n / np.linalg.norm(n)
    yh = np.cross(zh, xh)
    return xh, yh, zh, L0, (c - a) @ xh, (c - a) @ yh


def _pieces(o, a, b, c):
    """Local coordinates, vertex distances and the TMI term's half-Lambda /
    half-Omega, as the kernel has them before the gz step (float64)."""
    xh, yh, zh, L0, cx, cy = _frame(a, b, c)
    d = o - a
    x, y, z = d @ xh, d @ yh, d @ zh
    la = np.sqrt(x * x + y * y + z * z)
    lb = np.sqrt((L0 - x) ** 2 + y * y + z * z)
    lc = np.sqrt((cx - x) ** 2 + (cy - y) ** 2 + z * z)
    L1, L2 = np.hypot(cx - L0, cy), np.hypot(cx, cy)
    rbx, rcx, rcy = L0 - x, cx - x, cy - y
    den = la * lb * lc + (-x * rbx + y * y + z * z) * lc + (-x * rcx - y * rcy + z * z) * lb \
        + (rbx * rcx - y * rcy + z * z) * la
    om = np.arctan2(-z * L0 * cy, den)  # Omega / 2
    e = np.array([L0 / (la + lb), L1 / (lb + lc), L2 / (lc + la)])
    return dict(x=x, y=y, z=z, L0=L0, cx=cx, cy=cy, L1=L1, L2=L2, la=la, lb=lb, lc=lc, om=om, e=e)


def _quadrature(o, a, b, c, n=300):
    """int_F 1/|p - o| dA by the centroid rule on n^2 congruent sub-triangles."""
    A = 0.5 * np.linalg.norm(np.cross(b - a, c - a))
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = i + j < n
    pts = [((i[up] + 1 / 3) / n, (j[up] + 1 / 3) / n)]
    dn = i + j < n - 1
    pts.append(((i[dn] + 2 / 3) / n, (j[dn] + 2 / 3) / n))
    s = 0.0
    for u, v in pts:
        p = a + np.outer(u, b - a) + np.outer(v, c - a)
        s += (1.0 / np.linalg.norm(p - o, axis=1)).sum()
    return s * A / n ** 2


def _gauss_green(P):
    """I = sum_i u_i Lambda_i + z Omega (u_i: the station's projection to
    edge i's line, positive inside)."""
    x, y, z, L0, cx, cy, L1, L2 = (P[k] for k in ("x", "y", "z", "L0", "cx", "cy", "L1", "L2"))
    lam = 2.0 * np.arctanh(P["e"])
    u = [y, ((L0 - x) * cy + y * (cx - L0)) / L1, (x * cy - y * cx) / L2]
    return float(np.dot(u, lam) + z * 2.0 * P["om"])


def _regrouped(P, Q=None):
    """The kernel's mid-field form: I/2 = 2A/sbar + sum_i (u_i L_i / s_i)(Q_i +
    (sbar - s_i)/sbar) + z Omega/2, with the distance differences from their
    linear numerators."""
    x, y, z, L0, cx, cy = (P[k] for k in ("x", "y", "z", "L0", "cx", "cy"))
    la, lb, lc, e = P["la"], P["lb"], P["lc"], P["e"]
    if Q is None:
        Q = np.arctanh(e) / e - 1.0
    r0, r1, r2 = 1 / (la + lb), 1 / (lb + lc), 1 / (lc + la)
    k = 0.5 / (la + lb + lc)
    l2sq, l2l0sq, cxl0 = cx * cx + cy * cy, cx * cx + cy * cy - L0 * L0, cx - L0
    dba = L0 * (L0 - 2 * x) * r0
    dca = (l2sq - 2 * (cx * x + cy * y)) * r2
    dcb = (l2l0sq - 2 * (cxl0 * x + cy * y)) * r1
    w0, w1, w2 = y * L0 * r0, ((L0 - x) * cy + y * cxl0) * r1, (x * cy - y * cx) * r2
    h = w0 * (Q[0] + (dca + dcb) * k) + w1 * (Q[1] - (dba + dca) * k) + w2 * (Q[2] + (dba - dcb) * k)
    return 2.0 * (h + 3.0 * L0 * cy * k + z * P["om"])


def _atanh_q_any(e, dtype=np.float64):
    """The kernel's atanh_q_any: Q(e) = w^2 + (2 / (1 + c)) Q(w), c =
    sqrt(1 - e^2), w = e / (1 + c), until the series takes over at 0.2."""
    one, two = dtype(1), dtype(2)

    def series(v):
        v2 = v * v
        return v2 * (dtype(1 / 3) + v2 * (dtype(1 / 5) + v2 * (dtype(1 / 7) + v2 * dtype(1 / 9))))

    e = dtype(e)
    if not e > dtype(0.2):
        return series(e)
    q, m, v = dtype(0), one, e
    for _ in range(4):
        if not (v > dtype(0.2) and v < one):
            break
        r = one / (one + np.sqrt((one - v) * (one + v)))
        v = v * r
        q = q + m * v * v
        m = m * two * r
    if v <= dtype(0.2):
        return q + m * series(v)
    return dtype(0.5) * np.log1p(two * e / (one - e)) / e - one


@pytest.fixture(scope="module")
def pairs():
    """Seeded triangles with stations from 0.3 to 5 sizes off the centroid,
    above, below and in the facet plane's neighbourhood."""
    rng = np.random.default_rng(11)
    out = []
    for _ in range(40):
        a, b, c = (rng.normal(0.0, 50.0, 3) for _ in range(3))
        cen, size = (a + b + c) / 3, max(np.linalg.norm(b - a), np.linalg.norm(c - b), np.linalg.norm(a - c))
        d = rng.normal(size=3)
        ratio = rng.uniform(0.3, 5.0)
        o = cen + d / np.linalg.norm(d) * size * ratio
        out.append((o, a, b, c, ratio))
    return out


def test_gauss_green_form_is_the_facet_integral(pairs):
    for o, a, b, c, _ in pairs[:12]:
        want = _quadrature(o, a, b, c)
        got = _gauss_green(_pieces(o, a, b, c))
        assert abs(got - want) <= 2e-5 * abs(want), (got, want)  # the quadrature's own error


def test_regrouped_form_equals_gauss_green(pairs):
    for o, a, b, c, _ in pairs:
        P = _pieces(o, a, b, c)
        g = _gauss_green(P)
        assert abs(_regrouped(P) - g) <= 1e-12 * abs(g)


def test_half_argument_q_is_exact_and_does_not_cancel_in_fp32():
    """Q enters the mid-field sum as an absolute term next to the distance
    differences, so its absolute error is what counts."""
    e = np.concatenate([np.linspace(1e-4, 0.2, 200), np.linspace(0.2, 0.999, 800)])
    want = np.arctanh(e) / e - 1.0
    got64 = np.array([_atanh_q_any(v) for v in e])
    # the series' first omitted term, v^10/11, is below 1e-8 at v = 0.2; each
    # half-argument step at most doubles it, as it doubles atanh(e) / e
    assert np.max(np.abs(got64 - want) / (1.0 + want)) < 1e-8
    e32 = e.astype(np.float32)
    got32 = np.array([_atanh_q_any(v, np.float32) for v in e32], dtype=np.float64)
    want32 = np.arctanh(e32.astype(np.float64)) / e32 - 1.0
    err32 = np.abs(got32 - want32)
    assert np.max(err32 / (1.0 + want32)) < 3e-7  # a few FP32 ulp of atanh(e)/e, at every e
    # the direct "atanh(e)/e - 1" in FP32 carries atanh(e)/e's rounding (~1e-7)
    # into Q; the half-argument steps keep Q's own
    band = slice(200, 300)  # e in [0.2, 0.3]
    direct = np.array([np.float32(0.5) * np.log1p(np.float32(2) * v / (np.float32(1) - v)) / v - np.float32(1)
                       for v in e32[band]], dtype=np.float64)
    assert np.max(np.abs(direct - want32[band])) > 5 * np.max(err32[band])


def test_regrouped_form_with_kernel_q_in_fp32_keeps_ulp_level_error(pairs):
    """The regrouped mid-field gz with the kernel's Q, every input and step
    rounded to FP32, stays within a few 1e-7 of the facet integral from one
    facet size out (the mid field starts at tau/2 >= 1 size for the ratios
    the autotuner tries; nearer pairs are FP64), where the Gauss-Green sum
    written directly loses a factor distance / size."""
    f32 = np.float32
    worst_regrouped, worst_direct = 0.0, 0.0
    for o, a, b, c, ratio in pairs:
        if ratio < 1.0:
            continue
        P = _pieces(o, a, b, c)
        g = _gauss_green(P)
        P32 = {k: (v.astype(f32) if isinstance(v, np.ndarray) else f32(v)) for k, v in P.items()}
        Q32 = np.array([_atanh_q_any(v, f32) for v in P32["e"]], dtype=f32)
        r = float(_regrouped(P32, Q32))
        worst_regrouped = max(worst_regrouped, abs(r - g) / abs(g))
        lam32 = f32(2) * np.arctanh(P32["e"])
        x, y, z, L0, cx, cy, L1, L2 = (P32[k] for k in ("x", "y", "z", "L0", "cx", "cy", "L1", "L2"))
        u = np.array([y, ((L0 - x) * cy + y * (cx - L0)) / L1, (x * cy - y * cx) / L2], dtype=f32)
        d = float(np.dot(u, lam32) + z * f32(2) * P32["om"])
        worst_direct = max(worst_direct, abs(d - g) / abs(g))
    assert worst_regrouped < 1e-6
    assert worst_direct > worst_regrouped
