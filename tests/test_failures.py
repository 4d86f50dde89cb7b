"""Failure detection on the host, without a GPU.

The reference ignores damaged inputs (hercules_query_engine.c:2234 opens the
leaf file without checking; short reads go unnoticed) or exits the process.
This library returns a status code instead, and it checks the index files
before it touches a device, so these paths are exercised here on CPU: a
truncated leaves_raw.idx, a root.idx whose header or node records are
damaged, and a command-line query request beyond the query file."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HG_ERR_IO, HG_ERR_FORMAT = -2, -3


@pytest.fixture(scope="module")
def index_dir(oracle_mod, tmp_path_factory):
    """A small index in the reference's format, written by the oracle."""
    X = oracle_mod.gen_rows(1184, 3000, 64)
    oi = oracle_mod.OracleIndex.build(X, 400)
    d = str(tmp_path_factory.mktemp("idx")) + "/"
    oi.write(d, 64.0)
    return d


def _copy(src, tmp_path):
    d = str(tmp_path / "ix") + "/"
    shutil.copytree(src, d)
    return d


def _read_status(hg, d):
    with pytest.raises(hg.HerculesError) as e:
        hg.HerculesIndex.read(d)
    return e.value.status, str(e.value)


def test_truncated_leaf_file_is_an_io_error(hg, index_dir, tmp_path):
    d = _copy(index_dir, tmp_path)
    p = d + "leaves_raw.idx"
    size = os.path.getsize(p)
    with open(p, "r+b") as f:
        f.truncate(size - 4 * 64 * 7)  # seven rows short
    st, msg = _read_status(hg, d)
    assert st == HG_ERR_IO and "shorter" in msg


def test_missing_leaf_file_is_an_io_error(hg, index_dir, tmp_path):
    d = _copy(index_dir, tmp_path)
    os.remove(d + "leaves_raw.idx")
    assert _read_status(hg, d)[0] == HG_ERR_IO


@pytest.mark.parametrize("offset,value", [(24, 15), (28, 4), (16, 0), (16, 40)])
def test_damaged_header_is_a_format_error(hg, index_dir, tmp_path, offset, value):
    """paa_segments (24) not 16, sax_bit_cardinality (28) not 8, series length
    (16) zero or not a multiple of 16."""
    d = _copy(index_dir, tmp_path)
    with open(d + "root.idx", "r+b") as f:
        f.seek(offset)
        f.write(np.int32(value).tobytes())
    assert _read_status(hg, d)[0] == HG_ERR_FORMAT


def test_truncated_node_records_are_a_format_error(hg, index_dir, tmp_path):
    d = _copy(index_dir, tmp_path)
    p = d + "root.idx"
    with open(p, "r+b") as f:
        f.truncate(os.path.getsize(p) // 2)
    assert _read_status(hg, d)[0] == HG_ERR_FORMAT


def test_leaf_positions_out_of_order_are_a_format_error(hg, oracle_mod, tmp_path):
    """A leaf's file_pos must be where the DFS order puts it in
    leaves_raw.idx.  In a one-leaf index the root is the leaf and the last 8
    bytes of root.idx are its file_pos."""
    X = oracle_mod.gen_rows(1184, 300, 64)
    oi = oracle_mod.OracleIndex.build(X, 400)
    d = str(tmp_path / "one") + "/"
    os.makedirs(d)
    oi.write(d, 64.0)
    p = d + "root.idx"
    with open(p, "r+b") as f:
        f.seek(-8, os.SEEK_END)
        pos = np.frombuffer(f.read(8), np.uint64)[0]
        f.seek(-8, os.SEEK_END)
        f.write(np.uint64(pos + 1).tobytes())
    assert _read_status(hg, d)[0] == HG_ERR_FORMAT


def _cli(hg, *args):
    from hercules_b200 import build as B
    cli = B.build_cli()
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=120)


def test_cli_refuses_more_queries_than_the_file_holds(hg, index_dir, tmp_path):
    q = str(tmp_path / "q.bin")
    np.zeros((3, 64), np.float32).tofile(q)
    r = _cli(hg, "--mode", "1", "--serial", "1", "--num-threads", "1", "--k", "1", "--queries", q,
             "--queries-size", "5", "--index-path", index_dir)
    assert r.returncode == 1
    assert "has only 3 records" in r.stderr
    r = _cli(hg, "--mode", "1", "--serial", "1", "--num-threads", "1", "--k", "1", "--queries", q,
             "--queries-size", "2", "--queries-skip", "2", "--index-path", index_dir)
    assert r.returncode == 1 and "has only 3 records" in r.stderr


def test_cli_reports_a_missing_query_file(hg, index_dir, tmp_path):
    r = _cli(hg, "--mode", "1", "--serial", "1", "--num-threads", "1", "--k", "1", "--queries",
             str(tmp_path / "absent.bin"), "--queries-size", "1", "--index-path", index_dir)
    assert r.returncode == 1 and "not found" in r.stderr
