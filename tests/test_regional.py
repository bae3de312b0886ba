"""Regional systems on the CPU: the window search and moves of the oracle
against answers worked out by hand from SymPhas's formulas
(datatypes/inc/gridfunctions.h), and the library's host search
(sp_region_search, no GPU needed) against the oracle's on random windows."""
import numpy as np
import pytest

from oracle import spo
import symphas_b200 as sp

BD = 3


def _blob_buffer(d, cells):
    """Window buffer (rim included, x-fastest) with 1.0 at interior-local cells."""
    buf = np.zeros(tuple(reversed(d)))
    for c in cells:
        buf[tuple(reversed([x + BD for x in c]))] = 1.0
    return buf


def test_whole_domain_search_grows_the_box_and_pads_it():
    # get_view_resized_periodic: box x 10..14, y 5..8 -> origin (10, 5), dims
    # (5 + 6, 4 + 6); resize_adjust_region with factor 2: dims (22, 20), origin
    # 10 - (22 - 11) / 2 = 5 and 5 - (20 - 10) / 2 = 0
    G = (38, 38)
    cells = [(x, y) for x in range(10, 15) for y in range(5, 9)]
    buf = _blob_buffer(G, cells)
    assert spo.reg_search(2, G, (0, 0), G, buf, 0.5, 1, 2.0, 0.0) == ((5, 0), (22, 20))


def test_whole_domain_search_wraps_across_the_periodic_edge():
    # columns 30, 31, 0, 1 of a 32-wide domain: the box grows left from x = 0
    # through the edge to -2, so origin -2, width 4 + 6; padded to 20 the
    # origin -2 - 5 = -7 wraps to 25
    G = (38, 38)
    cells = [(x, y) for x in (30, 31, 0, 1) for y in range(5, 9)]
    buf = _blob_buffer(G, cells)
    assert spo.reg_search(2, G, (0, 0), G, buf, 0.5, 1, 2.0, 0.0) == ((25, 0), (20, 20))


def test_resize_keeps_dims_within_relative_tolerance():
    # window (4, 4) + dims (26, 26) holding a box x 8..13, y 9..14 of its
    # interior (positions 11..16, 12..17 with the rim): get_view_resized gives
    # origin (8 + 4, 9 + 4), dims (12, 12); doubled to 24, |24 - 26| / 26 < 0.1
    # keeps 26 and centres: origin 12 - (26 - 12) / 2 = 5 and 13 - 7 = 6
    G, o, d = (70, 70), (4, 4), (26, 26)
    cells = [(x, y) for x in range(8, 14) for y in range(9, 15)]
    buf = _blob_buffer(d, cells)
    assert spo.reg_search(2, G, o, d, buf, 0.5, 1, 2.0, 0.1) == ((5, 6), (26, 26))
    # with no tolerance the window takes the new dims: origin 12 - 6 = 6, 13 - 6 = 7
    assert spo.reg_search(2, G, o, d, buf, 0.5, 1, 2.0, 0.0) == ((6, 7), (24, 24))


def test_recentre_reads_buffer_entries_in_order():
    # get_view reads buffer entries 0 .. len(interior) - 1 at positions
    # (n / stride) % interior_dims: one value >= cutoff at buffer entry n
    # gives interval [p, p] per axis; with region dims 16 (interior 10) and n =
    # 3 + 16 * 5 = 83: x = 83 % 10 = 3, y = (83 / 16) % 10 = 5; dims 1 + 6 = 7,
    # delta = 16 - 7 = 9, origin = o + p - 4
    G, o, d = (40, 40), (7, 9), (16, 16)
    buf = np.zeros((16, 16))
    buf.ravel()[83] = 1.0
    assert spo.reg_search(2, G, o, d, buf, 0.5, 0) == ((7 + 3 - 4, 9 + 5 - 4), d)


def test_shift_in_place_takes_the_empty_test_from_the_last_axis():
    # adjust_origin_to_from, in place: shifting x by +5 (y unchanged) sets no
    # cell empty (the test reads the last axis, y, whose shift is 0); the cells
    # at the right end of each row take the buffer value 5 entries further on,
    # i.e. the rim and then the next row's first cells
    n = (20, 20)
    d = spo.make_desc(2, n, spo.MODEL_A, 1.0, 0.01, coeff=(1, 1))
    field = np.arange(400, dtype=np.float64).reshape(20, 20) + 1000.0
    r = spo.Regional(d, field)
    r.adjust((2, 3), (16, 14))  # a fresh window: interior 10 x 8, rim = empty 0
    win = r.get()
    assert win[3, 2] == field[3, 2] and win[2, 2] == 0.0
    buf = np.zeros((14, 16))
    buf[3:11, 3:13] = field[3:11, 2:12]
    r.adjust((7, 3), (16, 14))
    got = r.get()
    flat = buf.ravel()
    for y in range(8):
        for x in range(10):
            src = (x + 3) + (y + 3) * 16 + 5
            assert got[3 + y, (7 + x) % 20] == flat[src]
    # a shift along y (the last axis) empties what leaves
    r2 = spo.Regional(d, field)
    r2.adjust((2, 3), (16, 14))
    r2.adjust((2, 5), (16, 14))
    g2 = r2.get()
    assert g2[5, 2] == field[5, 2] and g2[11, 2] == 0.0 and g2[12, 2] == 0.0


def test_regional_oracle_steps_only_the_window():
    n = 48
    d = spo.make_desc(2, (n, n), spo.MODEL_A, 1.0, 0.01, coeff=(1, 1))
    y, x = np.mgrid[0:n, 0:n]
    f = np.where((x - 20) ** 2 + (y - 24) ** 2 < 36, 1.0, -1.0)
    r = spo.Regional(d, f, resize_delta=0.05)
    r.step(12)
    o, dims, empty, cutoff, t, nxt = r.window()
    assert empty == -1.0 and cutoff == -1.0 + 1e-6
    assert nxt == 3 and abs(t - 0.12) < 1e-12
    g = r.get()
    inside = np.zeros_like(g, dtype=bool)
    for j in range(dims[1] - 6):
        for i in range(dims[0] - 6):
            inside[(o[1] + j) % n, (o[0] + i) % n] = True
    assert np.all(g[~inside] == empty)
    # the window's interior holds what a full-domain run with the same rim
    # would give there: the blob evolved, values between the phases
    assert g[inside].max() > 0.9 and g[inside].min() >= -1.0


@pytest.mark.parametrize("D", [2, 3])
def test_library_search_matches_oracle_on_random_windows(D):
    rng = np.random.default_rng(11 + D)
    for _ in range(150):
        n = [int(rng.integers(8, 30)) for _ in range(D)]
        G = [v + 6 for v in n]
        if rng.random() < 0.3:
            o, d = [0] * D, list(G)
        else:
            d = [int(rng.integers(8, g + 1)) for g in G]
            o = [int(rng.integers(-3, g)) for g in G]
        shape = tuple(reversed(d))
        buf = np.zeros(shape)
        idx = np.indices(shape)
        for _ in range(int(rng.integers(0, 3))):
            c = [rng.integers(0, s) for s in shape]
            rad = rng.integers(1, 5)
            buf[sum((idx[i] - c[i]) ** 2 for i in range(D)) < rad * rad] = 1.0
        mask = (buf >= 0.5).astype(np.uint8)
        for mode in (0, 1):
            f = float(rng.choice([1.0, 1.5, 2.0]))
            eps = float(rng.choice([0.0, 0.05]))
            assert spo.reg_search(D, G, o, d, buf, 0.5, mode, f, eps) == \
                sp.region_search(D, G, o, d, mask, mode, f, eps)


def test_regional_create_rejects_without_a_gpu():
    # argument checks come before any device call: they run on any machine
    import ctypes

    from symphas_b200 import _capi as C

    def desc(**kw):
        d = C.SpDesc()
        d.dim, d.dtype, d.model, d.form = 2, C.SP_F64, C.SP_MODEL_A, C.SP_FORM_EXACT
        d.n[0], d.n[1], d.n[2] = 32, 32, 1
        d.lap_pts, d.gradlap_pts, d.bilap_pts = 5, 6, 13
        d.h, d.dt, d.batch, d.accuracy = 1.0, 0.01, 1, 2
        for k, v in kw.items():
            setattr(d, k, v)
        return d

    p = C.SpRegionalParams()
    p.resize_delta, p.padding_factor, p.cutoff_eps, p.fixed = 3.0, 2.0, 1e-6, 1
    out = ctypes.c_void_p()
    L = C.lib()
    cases = [desc(model=C.SP_MODEL_C), desc(batch=2), desc(dim=4)]
    d_dir = desc()
    d_dir.boundary[0] = C.SP_DIRICHLET
    cases.append(d_dir)
    for d in cases:
        assert L.sp_regional_create(ctypes.byref(d), ctypes.byref(p), ctypes.byref(out)) == C.SP_EINVAL
        assert L.sp_regional_error(None)
        assert not out.value
    bad = C.SpRegionalParams()
    bad.resize_delta, bad.padding_factor, bad.cutoff_eps = 0.0, 2.0, 1e-6
    assert L.sp_regional_create(ctypes.byref(desc()), ctypes.byref(bad), ctypes.byref(out)) == C.SP_EINVAL
    assert b"resize_delta" in L.sp_regional_error(None)
