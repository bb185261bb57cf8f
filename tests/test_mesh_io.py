"""The host-side mesh readers (no GPU): the .mesh / .bb text read one thread
per chunk of each section gives the generator's arrays bit for bit, text that
is not one record per line goes through the token reader with the same
result, the binary form reads back the same arrays, and malformed files are
TRN_ERR_IO (the reference's loader, io.cpp:53-161, asserts or reads garbage)."""
import os

import numpy as np
import pytest

from tests.oracle_lib import tags_of
from trinity_b200 import meshgen

ERR_IO = 2


def _read(mp, bp=None):
    from trinity_b200.api import read_mesh_files
    return read_mesh_files(mp, bp)


def _written(tmp_path, n=30):
    m, u, c = meshgen.make_config("c4", n)
    mp, bp = str(tmp_path / "a.mesh"), str(tmp_path / "a.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u)
    return m, u, mp, bp


def test_text_read_equals_the_arrays(tmp_path):
    m, u, mp, bp = _written(tmp_path)
    pts, tri, tags, uu = _read(mp, bp)
    assert np.array_equal(pts.view(np.uint64), np.ascontiguousarray(m.points).view(np.uint64))
    assert np.array_equal(tri, m.tris) and np.array_equal(tags, tags_of(m))
    assert np.array_equal(uu.view(np.uint64), np.ascontiguousarray(u).view(np.uint64))


def test_records_split_over_lines_read_the_same(tmp_path):
    m, u, mp, bp = _written(tmp_path, 12)
    txt = open(mp).read()
    head, rest = txt.split("Triangles\n", 1)
    cnt, body = rest.split("\n", 1)
    # every triangle record over two lines: the token reader's case
    lines = body.split("\n")
    nt = int(cnt)
    split = [" ".join(l.split()[:2]) + "\n" + " ".join(l.split()[2:]) for l in lines[:nt]]
    alt = str(tmp_path / "split.mesh")
    open(alt, "w").write(head + "Triangles\n" + cnt + "\n" + "\n".join(split) + "\n" + "\n".join(lines[nt:]))
    a = _read(mp, bp)
    b = _read(alt, bp)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_binary_form_reads_back(tmp_path):
    m, u, mp, bp = _written(tmp_path)
    pts, tri, tags, _ = _read(mp)
    binp = str(tmp_path / "a.trnb")
    hdr = np.zeros(8, np.int64)
    hdr[0] = int.from_bytes(b"TRNB0001", "little")
    hdr[1], hdr[2] = pts.shape[0], tri.shape[0]
    with open(binp, "wb") as f:
        f.write(hdr.tobytes() + pts.tobytes() + tags.tobytes() + tri.tobytes())
    p2, t2, g2, u2 = _read(binp, bp)
    assert np.array_equal(p2, pts) and np.array_equal(t2, tri) and np.array_equal(g2, tags)
    assert np.array_equal(u2, u)


@pytest.mark.parametrize("what", ["truncated_mesh", "bb_count", "missing"])
def test_malformed_files_are_io_errors(tmp_path, what):
    from trinity_b200.api import TrinityError
    m, u, mp, bp = _written(tmp_path, 10)
    if what == "truncated_mesh":
        txt = open(mp).read()
        open(mp, "w").write(txt[: txt.index("Triangles") + 60])
    elif what == "bb_count":
        meshgen.write_bb(bp, u[:-3])
    else:
        mp = str(tmp_path / "none.mesh")
    with pytest.raises(TrinityError) as e:
        _read(mp, bp)
    assert e.value.code == ERR_IO
