"""SymPhas's checkpoint text format (io/src/writegp.cpp:425-465, :780-806;
io/src/readgp.cpp:46-130): header and data layout, and a write/read round
trip at the ten digits the format keeps.  Host side only."""
import io

import numpy as np

from symphas_b200 import checkpoint as ck


def test_header_matches_the_printf_format():
    assert ck.header((64, 64), 0.5, 1000) == "2 64 64 0.000000 31.500000 0.000000 31.500000 1000 @\n"
    assert ck.header((8, 6, 4), 1.0, 0) == (
        "3 8 6 4 0.000000 7.000000 0.000000 5.000000 0.000000 3.000000 0 @\n")


def test_values_are_x_fastest_rows():
    a = np.array([[1.0, -2.5], [3.25e-7, 0.0]])
    assert ck.format_values(a) == (
        "1.0000000000E+00 -2.5000000000E+00 \n3.2500000000E-07 0.0000000000E+00 \n")


def test_round_trip_keeps_ten_digits():
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, size=(5, 7, 9))
    f = io.StringIO()
    ck.write(f, a, 1.0, 42)
    f.seek(0)
    index, dims, ends, b = ck.read(f)
    assert index == 42 and dims == [9, 7, 5] and ends[0] == (0.0, 8.0)
    assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(a))


def test_reader_skips_a_subdomain():
    text = "2 4 4 0.000000 3.000000 0.000000 3.000000 7 2 0.000000 1.000000 0.000000 1.000000\n"
    text += ck.format_values(np.arange(16.0).reshape(4, 4))
    index, dims, _, b = ck.read(io.StringIO(text))
    assert index == 7 and dims == [4, 4] and b[3, 3] == 15.0
