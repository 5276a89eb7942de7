"""XDMF output / checkpoint in the reference's format: the files this library writes equal, byte for byte, the
binary files of the reference's own XDMFOutput (geometry, topology, field data, checkpoint metadata) and describe
the same XML, and a checkpoint written here reads back exactly."""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import oracle as O
import ref as R
import terra_b200 as T

pytestmark = pytest.mark.gpu


def _fields(level, cuda):
    import torch

    sh = O.Shell(level)
    rng = np.random.default_rng(71)
    temp = rng.standard_normal(sh.scalar_shape)
    vel = rng.standard_normal(sh.vec_shape)
    return sh, temp, vel, torch.tensor(temp, device=cuda), torch.tensor(vel, device=cuda)


def _write_ours(tmp, level, t_dev, v_dev, geometry_bytes, out_bytes):
    g = T.Shell(level)
    w = T.XdmfWriter(g, 0, str(tmp), geometry_bytes=geometry_bytes)
    w.add("temperature", t_dev, out_bytes)
    w.add("velocity", v_dev, out_bytes)
    w.write()
    return g


def _xml_tree(path):
    root = ET.parse(path).getroot()

    def canon(e):
        return (e.tag, tuple(sorted(e.attrib.items())), (e.text or "").strip(), tuple(sorted(canon(c) for c in e)))

    return canon(root)


@pytest.mark.parametrize("geometry_bytes,out_bytes", [(4, 4), (8, 8)])
def test_xdmf_roundtrip(cuda, tmp_path, geometry_bytes, out_bytes):
    import torch

    level = 3
    sh, temp, vel, t_dev, v_dev = _fields(level, cuda)
    g = _write_ours(tmp_path / "ours", level, t_dev, v_dev, geometry_bytes, out_bytes)
    files = set(os.listdir(tmp_path / "ours"))
    assert {"geometry.bin", "topology.bin", "checkpoint_metadata.bin", "step_0.xmf", "temperature_0.bin",
            "velocity_0.bin"} <= files
    back_t = torch.zeros_like(t_dev)
    back_v = torch.zeros_like(v_dev)
    T.xdmf_read(g, 0, str(tmp_path / "ours"), "temperature", 0, back_t)
    T.xdmf_read(g, 0, str(tmp_path / "ours"), "velocity", 0, back_v)
    tol = 0.0 if out_bytes == 8 else 1e-7
    assert np.abs(back_t.cpu().numpy() - temp).max() <= tol * np.abs(temp).max()
    assert np.abs(back_v.cpu().numpy() - vel).max() <= tol * np.abs(vel).max()


@pytest.mark.skipif(not R.available(), reason="compiled reference (oracle/_ref) not present")
@pytest.mark.parametrize("geometry_bytes,out_bytes", [(4, 4), (8, 8)])
def test_xdmf_files_equal_reference(cuda, tmp_path, geometry_bytes, out_bytes):
    level = 3
    sh, temp, vel, t_dev, v_dev = _fields(level, cuda)
    _write_ours(tmp_path / "ours", level, t_dev, v_dev, geometry_bytes, out_bytes)
    R.xdmf_write(level, str(tmp_path / "ref"), temp, vel, geometry_bytes=geometry_bytes, out_bytes=out_bytes)
    for f in ("geometry.bin", "topology.bin", "checkpoint_metadata.bin", "temperature_0.bin", "velocity_0.bin"):
        a = (tmp_path / "ours" / f).read_bytes()
        b = (tmp_path / "ref" / f).read_bytes()
        assert a == b, f
    assert _xml_tree(tmp_path / "ours" / "step_0.xmf") == _xml_tree(tmp_path / "ref" / "step_0.xmf")
