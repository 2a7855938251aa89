"""The early exit of the CPIC particle fit (k_g2p_cdf) on the CPU.

The fit's 4x4 moment matrix Q = sum_i w_i p_i p_i^T (p_i = (dpt_i, 1), w_i the
B-spline weights of the nodes sharing an affinity with the particle) is
positive semi-definite, so det Q <= q00 q11 q22 q33 (Hadamard).  The kernel
skips the fit when that product times 1.01 is at most 1e-8, the threshold
below which the fit is declared singular (solver/g2p_cdf.rs:150-290).  Here
the same float32 operations (no multiply-add contraction, as the kernel is
built) run on random particles, cell widths and node subsets: the determinant
as the kernel evaluates it (2x2 minors) never exceeds 1.01 x the product, so
every skipped fit would have been singular."""
import numpy as np

F = np.float32


def _bspline(x):
    """Quadratic B-spline weights of the three stencil nodes for offset x in
    [0.5, 1.5] from the first node, in float32 (kernel_eval_all)."""
    x0, x1, x2 = F(x), F(x) - F(1), F(x) - F(2)
    w0 = F(0.5) * (F(1.5) - abs(x0)) * (F(1.5) - abs(x0))
    w1 = F(0.75) - x1 * x1
    w2 = F(0.5) * (F(1.5) - abs(x2)) * (F(1.5) - abs(x2))
    return [F(w0), F(w1), F(w2)]


def _det_minors(m):
    s0 = m[0][0] * m[1][1] - m[1][0] * m[0][1]
    s1 = m[0][0] * m[1][2] - m[1][0] * m[0][2]
    s2 = m[0][0] * m[1][3] - m[1][0] * m[0][3]
    s3 = m[0][1] * m[1][2] - m[1][1] * m[0][2]
    s4 = m[0][1] * m[1][3] - m[1][1] * m[0][3]
    s5 = m[0][2] * m[1][3] - m[1][2] * m[0][3]
    c5 = m[2][2] * m[3][3] - m[3][2] * m[2][3]
    c4 = m[2][1] * m[3][3] - m[3][1] * m[2][3]
    c3 = m[2][1] * m[3][2] - m[3][1] * m[2][2]
    c2 = m[2][0] * m[3][3] - m[3][0] * m[2][3]
    c1 = m[2][0] * m[3][2] - m[3][0] * m[2][2]
    c0 = m[2][0] * m[3][1] - m[3][0] * m[2][1]
    return s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0


def test_skipped_fits_are_singular():
    rng = np.random.default_rng(11)
    worst = 0.0
    skipped = 0
    for case in range(4000):
        dx = F([0.5, 0.25, 0.1, 1.0 / 32, 1.0 / 48, 1.0 / 64, 1.0 / 128][case % 7])
        off = rng.uniform(0.5, 1.5, 3).astype(F)  # particle offset from the first stencil node, in cells
        ref = [F(-o * dx) for o in off]
        w = [_bspline(o) for o in off]
        mask = rng.random(27) < rng.uniform(0.1, 1.0)  # nodes sharing an affinity with the particle
        q = [[F(0)] * 4 for _ in range(4)]
        for i in range(27):
            if not mask[i]:
                continue
            sx, sy, sz = i % 3, (i // 3) % 3, i // 9
            p = [F(ref[0] + F(sx) * dx), F(ref[1] + F(sy) * dx), F(ref[2] + F(sz) * dx), F(1)]
            wt = F(F(w[0][sx] * w[1][sy]) * w[2][sz])
            for r in range(4):
                for c in range(4):
                    q[r][c] = F(q[r][c] + F(F(p[r] * p[c]) * wt))
        hprod = F(F(F(F(q[0][0] * q[1][1]) * q[2][2]) * q[3][3]) * F(1.01))
        det = F(_det_minors(q))
        if hprod > 0:
            worst = max(worst, float(det) / float(hprod))
        assert det <= hprod or hprod == 0 and det <= F(1e-30), (case, det, hprod)
        if hprod <= F(1e-8):
            skipped += 1
            assert det <= F(1e-8)
    print("largest det / (1.01 x diagonal product):", worst, "skipped", skipped)
    assert skipped > 1000
