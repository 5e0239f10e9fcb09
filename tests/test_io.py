"""Readers of the reference's file formats (no GPU needed): the README
example files of the reference (README.md:57-96) under tests/golden/readme."""
import os

import numpy as np
import pytest

import sgs

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "readme")


def test_readme_graph_file():
    nv, src, dst, w = sgs.read_edge_list(os.path.join(HERE, "input.txt"))
    assert nv == 5 and w is None
    assert list(zip(src.tolist(), dst.tolist())) == [(0, 1), (0, 2), (1, 2), (1, 3), (2, 4), (3, 4)]


def test_readme_update_and_stream_size_files():
    adds, dels = sgs.read_stream_sizes(os.path.join(HERE, "stream_size.txt"))
    assert adds.tolist() == [2, 2] and dels.tolist() == [3, 3]
    u = sgs.read_update_file(os.path.join(HERE, "update.txt"))
    assert list(zip(u["add_u"].tolist(), u["add_v"].tolist())) == [(0, 3), (0, 4), (1, 4), (2, 3)]
    assert list(zip(u["del_u"].tolist(), u["del_v"].tolist())) == [
        (0, 1), (0, 2), (1, 2), (1, 3), (2, 4), (3, 4)]
    assert u["add_w"].tolist() == [0, 0, 0, 0]


def test_weights_comments_and_unknown_lines(tmp_path):
    g = tmp_path / "g.txt"
    g.write_text("# comment\n% also\n\n3 7 5\n  1 2 9\r\n")
    nv, src, dst, w = sgs.read_edge_list(g)
    assert nv == 8 and src.tolist() == [3, 1] and dst.tolist() == [7, 2] and w.tolist() == [5, 9]
    up = tmp_path / "u.txt"
    up.write_text("a 1 2 7\nx 5 5\nd 3 4\nadd 9 9\n")
    u = sgs.read_update_file(up)
    assert u["add_u"].tolist() == [1] and u["add_w"].tolist() == [7]
    assert u["del_u"].tolist() == [3] and u["del_w"].tolist() == [0]


def test_malformed_inputs_are_errors(tmp_path):
    g = tmp_path / "bad.txt"
    g.write_text("0 1\n2\n")
    with pytest.raises(sgs.SgsError) as e:
        sgs.read_edge_list(g)
    assert e.value.code == -1 and "line 2" in str(e.value)
    with pytest.raises(sgs.SgsError):
        sgs.read_edge_list(tmp_path / "missing.txt")
    s = tmp_path / "s.txt"
    s.write_text("2\n")
    with pytest.raises(sgs.SgsError):
        sgs.read_stream_sizes(s)
    big = tmp_path / "big.txt"
    big.write_text("0 4294967295\n")
    with pytest.raises(sgs.SgsError):
        sgs.read_edge_list(big)
