"""Membrane dumps in the reference's PLY layout (src/io/mesh/imp/main.h:52-134),
written by the library without a GPU and read back byte by byte."""
import numpy as np

from ctc_b200 import systems


def _read(path):
    data = open(path, "rb").read()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    return data[:end].decode(), data[end:]


def test_ply_layout(tmp_path):
    import ctc_b200 as C
    L = (24, 20, 16)
    pv, tri, par = systems.rbc_system(L, 2, seed=5)
    nv = len(pv) // 2
    tri = np.asarray(tri, np.int32)
    for shift, off in (("edge", np.float32([12, 10, 8])), ("center", np.float32([0, 0, 0]))):
        p = tmp_path / ("m_%s.ply" % shift)
        C.mesh_write_ply(p, pv, tri, nv, L, shift=shift)
        head, body = _read(p)
        assert head == ("ply\nformat binary_little_endian 1.0\nelement vertex %d\n"
                        "property float x\nproperty float y\nproperty float z\n"
                        "property float u\nproperty float v\nproperty float w\n"
                        "element face  %d\nproperty list int int vertex_index\nend_header\n"
                        % (2 * nv, 2 * len(tri)))
        nvb = 2 * nv * 6 * 4
        vert = np.frombuffer(body[:nvb], "<f4").reshape(-1, 6)
        faces = np.frombuffer(body[nvb:], "<i4").reshape(-1, 4)
        assert len(body) == nvb + 2 * len(tri) * 16
        assert np.array_equal(vert[:, :3], pv[:, :3] + off)
        assert np.array_equal(vert[:, 3:], pv[:, 3:])
        assert np.all(faces[:, 0] == 3)
        assert np.array_equal(faces[:len(tri), 1:], tri)
        assert np.array_equal(faces[len(tri):, 1:], tri + nv)


def test_ply_rejects_bad_triangles(tmp_path):
    import pytest
    import ctc_b200 as C
    pv, tri, par = systems.rbc_system((16, 16, 16), 1, seed=5)
    bad = np.asarray(tri, np.int32).copy()
    bad[3, 1] = len(pv)
    with pytest.raises(C.CtcError):
        C.mesh_write_ply(tmp_path / "bad.ply", pv, bad, len(pv), (16, 16, 16))
