"""Edge-list files in and per-vertex CSV out (plato_edge_list_read_csv,
plato_write_vertex_csv): the reference's csv_parser rules
(plato/graph/parsers.hpp:226-290), file listing (plato/graph/detail.hpp:82-108),
gzip handling (detail.hpp:196-212) and result layout
(example/pagerank.cc:191-200, plato/util/foutput.cc:95-101).  CPU only."""
import gzip

import numpy as np
import pytest

import plato_b200 as pb


def _write(path, text, gz=False):
    if gz:
        with gzip.open(path, "wb") as f:
            f.write(text.encode())
    else:
        path.write_text(text)


def test_csv_line_rules(tmp_path):
    # strtok: empty fields are skipped; strtoul: blanks and a sign before the
    # digits, the digits up to the first other character, no digits -> 0
    text = "0,1\n\n 2 , 3\n5\n,,4,,6\n7,8,9\n+1,2\r\nx,3\n10,\n"
    _write(tmp_path / "e.csv", text)
    V, s, d = pb.read_csv(tmp_path / "e.csv")
    assert s.tolist() == [0, 2, 4, 7, 1, 0]
    assert d.tolist() == [1, 3, 6, 8, 2, 3]
    assert V == 9


def test_csv_weighted_line_rules(tmp_path):
    # double_decoder (parsers.hpp:84-88): the third strtok field through
    # strtod; a line without one fails to decode and is skipped
    text = "0,1,2.5\n1,2\n 2 , 3 , 1e2\n,,4,,6,,-0.25,9\n5,6,abc\n7,8, \n7,8,0x10\n9,1,3"
    _write(tmp_path / "w.csv", text)
    V, s, d, w = pb.read_csv(tmp_path / "w.csv", weighted=True)
    assert s.tolist() == [0, 2, 4, 5, 7, 7, 9]
    assert d.tolist() == [1, 3, 6, 6, 8, 8, 1]
    assert w.tolist() == [2.5, 100.0, -0.25, 0.0, 0.0, 16.0, 3.0]
    assert V == 10
    # the unweighted reader ignores the third field
    V2, s2, d2 = pb.read_csv(tmp_path / "w.csv")
    assert s2.size == 8 and V2 == 10


def test_csv_last_line_without_newline_and_empty_file(tmp_path):
    _write(tmp_path / "a.csv", "3,4\n4,5")
    V, s, d = pb.read_csv(tmp_path / "a.csv")
    assert (s.tolist(), d.tolist(), V) == ([3, 4], [4, 5], 6)
    _write(tmp_path / "b.csv", "")
    V, s, d = pb.read_csv(tmp_path / "b.csv")
    assert V == 0 and s.size == 0 and d.size == 0


@pytest.mark.parametrize("bad", ["4294967296,1", "1,-2", "99999999999999999999999,1"])
def test_csv_id_out_of_range_is_an_error(tmp_path, bad):
    _write(tmp_path / "e.csv", "0,1\n" + bad + "\n")
    with pytest.raises(pb.PlatoError) as e:
        pb.read_csv(tmp_path / "e.csv")
    assert e.value.code == 1 and ":2:" in str(e.value)  # EINVAL, line 2


def test_csv_max_id_leaves_no_vertex_count(tmp_path):
    _write(tmp_path / "e.csv", "4294967295,0\n")
    with pytest.raises(pb.PlatoError):
        pb.read_csv(tmp_path / "e.csv")


def test_missing_path_is_an_error(tmp_path):
    with pytest.raises(pb.PlatoError):
        pb.read_csv(tmp_path / "nope.csv")


def test_reference_fixture_graphs_round_trip(tmp_path, golden):
    """The reference's fixture graphs, written as CSV in several spellings
    (plain, CRLF + blanks, gzip, split over a directory), read back equal."""
    graphs, _ = golden
    for name in ("graph_10_9", "v100_e2150_ua_c3", "v100_e4300_da_c3"):
        s0, d0 = graphs[name + ".csv"]["src"], graphs[name + ".csv"]["dst"]
        plain = "".join(f"{a},{b}\n" for a, b in zip(s0, d0))
        crlf = "".join(f" {a} ,{b}\r\n\n" for a, b in zip(s0, d0))
        _write(tmp_path / f"{name}.csv", plain)
        _write(tmp_path / f"{name}_crlf.csv", crlf)
        _write(tmp_path / f"{name}.csv.gz", plain, gz=True)
        part = tmp_path / f"{name}_dir"
        part.mkdir()
        half = len(s0) // 2
        _write(part / "part-0001.csv", "".join(f"{a},{b}\n" for a, b in zip(s0[half:], d0[half:])))
        _write(part / "part-0000.csv.gz", "".join(f"{a},{b}\n" for a, b in zip(s0[:half], d0[:half])),
               gz=True)
        for p in (f"{name}.csv", f"{name}_crlf.csv", f"{name}.csv.gz", f"{name}_dir"):
            V, s, d = pb.read_csv(tmp_path / p)
            np.testing.assert_array_equal(s, s0)
            np.testing.assert_array_equal(d, d0)
            assert V == int(max(s0.max(), d0.max())) + 1


def test_large_file_parses_in_parallel_pieces(tmp_path):
    rng = np.random.default_rng(7)
    n = 600_000  # several MiB: the parser cuts the buffer into per-thread pieces
    s0 = rng.integers(0, 1 << 31, n, dtype=np.uint64).astype(np.uint32)
    d0 = rng.integers(0, 1 << 20, n, dtype=np.uint64).astype(np.uint32)
    lines = np.char.add(np.char.add(s0.astype(str), ","), d0.astype(str))
    (tmp_path / "big.csv").write_text("\n".join(lines.tolist()) + "\n")
    V, s, d = pb.read_csv(tmp_path / "big.csv")
    np.testing.assert_array_equal(s, s0)
    np.testing.assert_array_equal(d, d0)
    assert V == int(max(s0.max(), d0.max())) + 1


@pytest.mark.parametrize("gz", [False, True])
def test_write_vertex_csv_layout(tmp_path, gz):
    vals = np.array([0.5, 1e-7, 3.0, 0.15000000596, 2.5e6], np.float32)
    pb.write_vertex_csv(tmp_path, vals, prefix="0000_", files=2, gzip=gz)
    ext = ".csv.gz" if gz else ".csv"
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == [f"0000_0000{ext}", f"0000_0001{ext}"]
    text = ""
    for nm in names:
        raw = (gzip.open(tmp_path / nm).read() if gz else (tmp_path / nm).read_bytes()).decode()
        text += raw
    want = "".join("%d,%g\n" % (v, float(x)) for v, x in enumerate(vals))
    assert text == want
    first = (gzip.open(tmp_path / names[0]).read() if gz else (tmp_path / names[0]).read_bytes()).decode()
    assert first.splitlines()[0] == "0,0.5" and len(first.splitlines()) == 2  # vertices [0, 2)


def test_write_vertex_csv_integers_and_errors(tmp_path):
    lev = np.array([0, 1, pb.PLATO_LEVEL_UNREACHED, 2], np.uint32)
    pb.write_vertex_csv(tmp_path, lev, files=1)
    assert (tmp_path / "0000.csv").read_text() == "0,0\n1,1\n2,%d\n3,2\n" % pb.PLATO_LEVEL_UNREACHED
    with pytest.raises(TypeError):
        pb.write_vertex_csv(tmp_path, np.zeros(3, np.float64))
    with pytest.raises(pb.PlatoError):
        pb.write_vertex_csv(tmp_path / "missing_dir", lev)
    with pytest.raises(pb.PlatoError):
        pb.write_vertex_csv(tmp_path, lev, files=0)
