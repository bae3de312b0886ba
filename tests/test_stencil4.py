"""The oracle's 4th-order 2D stencils (Stencil2d4h, sol/inc/stencilh4.h),
pinned without the reference's build: known answers on polynomials at h = 1
for every consistent point set, the reference's scale factor (divh3 for all
three operators, sol/inc/stencilincludes.h:446-460) at h != 1, and an
independent NumPy transcription of every point set -- including the
gradlaplacians <18>, <26> and <30>, whose x, x2 and x3 terms the reference
writes one-sided (stencilh4.h:165-216), so they approximate no derivative;
that is kept as the reference's behaviour."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import spo  # noqa: E402

import symphas_b200 as sp  # noqa: E402

N = 24
_y, _x = np.mgrid[0:N, 0:N].astype(float)
X, Y = _x - 11.3, _y - 12.1
INNER = (slice(3, N - 3), slice(3, N - 3))  # three cells from the periodic seam
# f, lap f, bilap f, d/dx lap f
POLYS = [
    (X ** 4 + X ** 2 * Y ** 2 - 2 * Y ** 4 + X ** 3 * Y,
     14 * X ** 2 + 6 * X * Y - 22 * Y ** 2, -16 + 0 * X, 28 * X + 6 * Y),
    (X ** 5, 20 * X ** 3, 120 * X, 60 * X ** 2),
    (X ** 3 * Y ** 2, 6 * X * Y ** 2 + 2 * X ** 3, 24 * X, 6 * Y ** 2 + 6 * X ** 2),
]
OPID = {"lap": spo.OP_LAP, "bilap": spo.OP_BILAP, "gradlap": spo.OP_GRADLAP}


def rhs4(op, pts, f, h=1.0):
    return spo.rhs(spo.make_desc(2, (N, N), OPID[op], h, 0.0, stencil=pts, acc=4), f)


def rel(a, b):
    return float(np.max(np.abs(a[INNER] - b[INNER])) / max(1.0, np.max(np.abs(b[INNER]))))


@pytest.mark.parametrize("op,pts", [("lap", (9, 14, 21)), ("lap", (17, 14, 21)),
                                    ("lap", (21, 14, 21)), ("bilap", (9, 14, 21)),
                                    ("bilap", (9, 14, 25)), ("bilap", (9, 14, 33)),
                                    ("bilap", (9, 14, 37)), ("gradlap", (9, 14, 21))])
def test_fourth_order_stencils_are_exact_on_polynomials(op, pts):
    k = {"lap": 1, "bilap": 2, "gradlap": 3}[op]
    for poly in POLYS:
        assert rel(rhs4(op, pts, poly[0]), poly[k]) < 1e-10, (op, pts)


def test_reference_scale_factor_divh3():
    """At h = 0.5 the reference's Laplacian comes out 1/h = 2 times too large
    and its bilaplacian h = 0.5 times too small; the gradlaplacian, given the
    divh3 it expects, is right."""
    h = 0.5
    f, lap, bilap, glap = POLYS[0]
    fh = f  # values on the grid; derivatives in grid units scale by 1/h^k
    assert rel(rhs4("lap", (9, 14, 21), fh, h), lap / h ** 2 * (1 / h)) < 1e-10
    assert rel(rhs4("bilap", (9, 14, 21), fh, h), bilap / h ** 4 * h) < 1e-10
    assert rel(rhs4("gradlap", (9, 14, 21), fh, h), glap / h ** 3) < 1e-10


def _np_stencils(v, s):
    """The point sets of sol/inc/stencilh4.h in NumPy, on a periodic grid."""
    def P(i, j):
        return np.roll(np.roll(v, -i, axis=1), -j, axis=0)
    vx, vx_, vy, vy_ = P(1, 0), P(-1, 0), P(0, 1), P(0, -1)
    vx2, vx2_, vy2, vy2_ = P(2, 0), P(-2, 0), P(0, 2), P(0, -2)
    vx3, vx3_, vy3, vy3_ = P(3, 0), P(-3, 0), P(0, 3), P(0, -3)
    vxy, vx_y, vxy_, vx_y_ = P(1, 1), P(-1, 1), P(1, -1), P(-1, -1)
    vx2y, vx2_y, vx2y_, vx2_y_ = P(2, 1), P(-2, 1), P(2, -1), P(-2, -1)
    vxy2, vx_y2, vxy2_, vx_y2_ = P(1, 2), P(-1, 2), P(1, -2), P(-1, -2)
    vx2y2, vx2_y2, vx2y2_, vx2_y2_ = P(2, 2), P(-2, 2), P(2, -2), P(-2, -2)
    vx3y, vx3_y, vx3y_, vx3_y_ = P(3, 1), P(-3, 1), P(3, -1), P(-3, -1)
    vxy3, vx_y3, vxy3_, vx_y3_ = P(1, 3), P(-1, 3), P(1, -3), P(-1, -3)
    vx3y3, vx3_y3, vx3y3_, vx3_y3_ = P(3, 3), P(-3, 3), P(3, -3), P(-3, -3)
    v0 = v
    lap = {
        9: (-vx2_ - vx2 - vy2 - vy2_ + 16. * (vx_ + vx + vy + vy_) - 60. * v0) * s / 12,
        17: (-(vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) - 8. * (vx2 + vx2_ + vy2 + vy2_)
             + 16. * (vxy + vx_y + vxy_ + vx_y_) + 128. * (vx + vx_ + vy + vy_) - 540. * v0) * s / 120,
        21: (-2. * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_)
             - (vx2 + vx2_ + vy2 + vy2_) + 16. * (vxy + vx_y + vxy_ + vx_y_)
             + 52. * (vx + vx_ + vy + vy_) - 252. * v0) * s / 60}
    bilap = {
        21: (-4. * (vx3 + vx3_ + vy3 + vy3_) - (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_)
             + 50. * (vx2 + vx2_ + vy2 + vy2_) + 64. * (vxy + vx_y + vxy_ + vx_y_)
             - 284. * (vx + vx_ + vy + vy_) + 700. * v0) * s / 24,
        25: (-(vx3 + vx3_ + vy3 + vy3_) - (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_)
             + 14. * (vx2 + vx2_ + vy2 + vy2_) + 20. * (vxy + vx_y + vxy_ + vx_y_)
             - 77. * (vx + vx_ + vy + vy_) + 184. * v0) * s / 6,
        33: (-17. * (vx3y3 + vx3_y3 + vx3y3_ + vx3_y3_) - 236. * (vx3 + vx3_ + vy3 + vy3_)
             + 351. * (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_)
             - 756. * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_)
             + 4050. * (vx2 + vx2_ + vy2 + vy2_) + 5049. * (vxy + vx_y + vxy_ + vx_y_)
             - 19116. * (vx + vx_ + vy + vy_) + 45724. * v0) * s / 1620,
        37: (-17. * (vx3y + vx3_y + vx3y_ + vx3_y_ + vxy3 + vx_y3 + vxy3_ + vx_y3_)
             + 4. * (vx3 + vx3_ + vy3 + vy3_) - 29. * (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_)
             + 188. * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_)
             + 42. * (vx2 + vx2_ + vy2 + vy2_) - 374. * (vxy + vx_y + vxy_ + vx_y_)
             - 764. * (vx + vx_ + vy + vy_) + 3116. * v0) * s / 180}
    grad = {
        14: (-6. * (vx3 - vx3_) - (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + 50. * (vx2 - vx2_)
             + 32. * (vxy - vx_y + vxy_ - vx_y_) - 142. * (vx - vx_)) * s / 48,
        18: (-3. * vx3 - 2. * (vx2y - vx2_y + vx2y_ - vx2_y_) + 28. * vx2
             - (vxy2 - vx_y2 + vxy2_ - vx_y2_) + 20. * (vxy - vx_y + vxy_ - vx_y_) - 77. * vx) * s / 24,
        26: (-17. * (vx3y3 - vx3_y3 + vx3y3_ - vx3_y3_) - 236. * vx3
             + 234. * (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) - 504. * (vx2y - vx2_y + vx2y_ - vx2_y_)
             + 2700. * vx2 - 252. * (vxy2 - vx_y2 + vxy2_ - vx_y2_)
             + 1683. * (vxy - vx_y + vxy_ - vx_y_) - 6372. * vx) / (2160. * s),
        30: (-51. * (vx3y - vx3_y + vx3y_ - vx3_y_) + 12. * vx3
             - 58. * (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + 376. * (vx2y - vx2_y + vx2y_ - vx2_y_)
             + 84. * vx2 - 17. * (vxy3 - vx_y3 + vxy3_ - vx_y3_)
             + 188. * (vxy2 - vx_y2 + vxy2_ - vx_y2_) - 374. * (vxy - vx_y + vxy_ - vx_y_)
             - 764. * vx) * s / 720}
    return lap, bilap, grad


def test_every_fourth_order_point_set_matches_an_independent_transcription():
    h = 0.7
    s = (1 / h) ** 3
    v = spo.seed_uniform(5, -1.0, 1.0, N * N).reshape(N, N)
    lap, bilap, grad = _np_stencils(v, s)
    for L in (9, 17, 21):
        assert np.allclose(rhs4("lap", (L, 14, 21), v, h), lap[L], rtol=1e-12, atol=1e-12)
    for B in (21, 25, 33, 37):
        assert np.allclose(rhs4("bilap", (9, 14, B), v, h), bilap[B], rtol=1e-12, atol=1e-10)
    for G in (14, 18, 26, 30):
        assert np.allclose(rhs4("gradlap", (9, G, 21), v, h), grad[G], rtol=1e-12, atol=1e-10)


def test_stencil2d4h_reaches_the_description():
    st = sp.Stencil2d4h()
    assert st.points == (9, 14, 21) and st.accuracy == 4 and st.dim == 2
    assert sp.Stencil2d2h().accuracy == 2 and sp.Stencil3d2h().accuracy == 2
