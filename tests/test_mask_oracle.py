"""The mask-generator oracle (oracle/mask_ref.c) against the reference's own
known-answer and metamorphic tests for mask.polygon@1
(crates/paintop-cpu/src/mask_polygon/tests.rs) and mask.ellipse@1
(crates/paintop-cpu/src/ellipse/tests.rs), restated with the same inputs and
bars."""
import math

import numpy as np

from oracle import oracle as O

TOL = 1e-9


# ---- mask.polygon@1 ---------------------------------------------------------
def test_integer_square_is_hard_half_open():  # mask_polygon/tests.rs:67-85
    s = O.mask_polygon(6, 6, [[1, 1], [4, 1], [4, 4], [1, 4]], "nonzero")
    want = np.zeros((6, 6), np.float32)
    want[1:4, 1:4] = 1.0
    assert np.array_equal(s.view(np.uint32), want.view(np.uint32))


def _triangle_area_at(scale, size):  # mask_polygon/tests.rs:91-103
    pts = [[x * scale, y * scale] for x, y in [(1.0, 1.0), (7.0, 2.0), (3.0, 7.0)]]
    return float(O.mask_polygon(size, size, pts).astype(np.float64).sum()) / (scale * scale)


def test_area_converges_to_analytic_with_resolution():  # :105-119
    coarse = abs(_triangle_area_at(1.0, 8) - 17.0)
    fine = abs(_triangle_area_at(8.0, 64) - 17.0)
    assert fine < coarse and fine < 0.5


def _pentagram(c, r):  # :123-137 (its fused multiply-adds as two roundings: only
    pts = []            # inside / outside at the centre is asserted)
    for k in range(5):
        theta = k * 2.0 * (2.0 * math.pi / 5.0) - math.pi / 2.0
        pts.append([r * math.cos(theta) + c, r * math.sin(theta) + c])
    return pts


def test_fill_rule_changes_pentagram_centre():  # :139-179
    pts = _pentagram(20.0, 15.0)
    nz = O.mask_polygon(40, 40, pts, "nonzero")
    eo = O.mask_polygon(40, 40, pts, "even-odd")
    assert nz[20, 20] > 0.5 and eo[20, 20] < 0.5
    assert nz.astype(np.float64).sum() > eo.astype(np.float64).sum()


def test_degenerate_edges_produce_finite_coverage():  # :181-210
    for pts in ([[1, 1], [1, 1], [5, 1], [5, 5], [1, 5]], [[1, 1], [3, 1], [5, 1], [5, 5], [1, 5]],
                [[0, 0], [6, 6], [6, 0], [0, 6]], [[1, 1], [5, 1], [3, 1], [3, 5]], [[1, 1], [4, 4]]):
        for rule in ("nonzero", "even-odd"):
            s = O.mask_polygon(8, 8, pts, rule)
            assert np.isfinite(s).all() and (s >= 0).all() and (s <= 1).all()


def test_fewer_than_three_vertices_is_empty():  # :212-216
    s = O.mask_polygon(6, 6, [[1, 1], [4, 4]])
    assert not s.view(np.uint32).any()


def test_rotation_covariance():  # :218-257
    n = 16
    base_pts = [(3.0, 2.0), (12.0, 4.0), (6.0, 13.0)]
    rot_pts = [(n - y, x) for x, y in base_pts]
    base = O.mask_polygon(n, n, base_pts)
    rotated = O.mask_polygon(n, n, rot_pts)
    # out(x, y) = in(y, n - 1 - x)
    yy, xx = np.mgrid[0:n, 0:n]
    base_then_rotated = base[n - 1 - xx, yy]
    assert np.array_equal(rotated.view(np.uint32), base_then_rotated.view(np.uint32))


# ---- mask.ellipse@1 ---------------------------------------------------------
def test_coverage_is_bounded_and_finite():  # ellipse/tests.rs:88-103
    m = O.mask_ellipse(64, 64, (33.0, 24.0), (18.0, 7.0), 0.6, 3.0)
    assert np.isfinite(m).all() and (m >= 0).all() and (m <= 1).all()


def test_rendered_area_converges_to_analytic_area():  # :105-133
    rx, ry = 0.30, 0.18
    analytic = math.pi * rx * ry
    prev = math.inf
    for n in (64, 128, 256):
        m = O.mask_ellipse(n, n, (n / 2.0, n / 2.0), (rx * n, ry * n))
        err = abs(float(m.astype(np.float64).sum()) / (n * n) - analytic)
        assert err < prev + 1e-4
        prev = err
    assert prev < 1e-3


def test_circle_is_invariant_under_ninety_degree_rotation():  # :135-157
    a = O.mask_ellipse(32, 32, (16.0, 16.0), (9.0, 9.0), 0.0, 2.0)
    b = O.mask_ellipse(32, 32, (16.0, 16.0), (9.0, 9.0), math.pi / 2, 2.0)
    assert np.abs(a.astype(np.float64) - b).max() < TOL


def test_quarter_turn_equals_swapping_radii():  # :159-178
    a = O.mask_ellipse(32, 32, (16.0, 16.0), (10.0, 4.0), math.pi / 2)
    b = O.mask_ellipse(32, 32, (16.0, 16.0), (4.0, 10.0), 0.0)
    assert np.abs(a.astype(np.float64) - b).max() < TOL


def test_integer_translation_shifts_coverage():  # :180-213
    a = O.mask_ellipse(40, 40, (18.0, 18.0), (6.0, 9.0), 0.3, 2.0)
    b = O.mask_ellipse(40, 40, (22.0, 21.0), (6.0, 9.0), 0.3, 2.0)
    assert np.abs(a[:37, :36].astype(np.float64) - b[3:, 4:]).max() < TOL


def test_half_open_convention_on_pixel_aligned_boundary():  # :280-304
    m = O.mask_ellipse(17, 17, (8.5, 8.5), (4.0, 4.0))
    assert abs(float(m[8, 12]) - 1.0) < TOL and abs(float(m[8, 13])) < TOL


def test_feather_band_is_two_half_widths():  # :215-256, on pixel centres of a row
    # a circle of radius 200 centred at (0.5, 0.5): along row 0 the sample at pixel
    # i sits at distance i from the centre, on the boundary normal
    r, h = 200.0, 6.0
    m = O.mask_ellipse(220, 1, (0.5, 0.5), (r, r), 0.0, h)[0].astype(np.float64)
    assert abs(m[int(r - h)] - 1.0) < 1e-3 and abs(m[int(r + h)]) < 1e-3
    assert abs(m[int(r)] - 0.5) < 1e-3
    assert m[int(r - h) + 1] < 1.0 and m[int(r + h) - 1] > 0.0
    assert abs(m[int(r - h) - 1] - 1.0) < TOL and abs(m[int(r + h) + 1]) < TOL
