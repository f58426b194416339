"""Particle backups in the reference's Fortran unformatted format
(DATA.BAK/particlesNNN.bak, Src/main.f90:1294-1330, Src/restart.f90:62-70):
record framing and gfortran's subrecord split checked byte for byte on CPU;
save / restart of a device state on the GPU (FP64 bit for bit, mixed form to
FP32 rounding of the offsets)."""
import struct

import numpy as np
import pytest

from essaitemporaire_lepic_module_b200 import checkpoint
from tests.conftest import have_gpu


def test_record_layout_by_hand(tmp_path):
    path = tmp_path / "p.bak"
    v0 = np.arange(12, dtype=np.float64).reshape(2, 6)
    v1 = np.arange(6, dtype=np.float64).reshape(1, 6) + 100
    checkpoint.write_particles_bak(path, 1.5e-9, [2, 1], [v0, v1])
    raw = path.read_bytes()
    # four records: time, np_tot(2,1), 2x6 doubles, 1x6 doubles
    want = (struct.pack("<i", 8) + struct.pack("<d", 1.5e-9) + struct.pack("<i", 8)
            + struct.pack("<iiii", 8, 2, 1, 8)
            + struct.pack("<i", 96) + v0.tobytes() + struct.pack("<i", 96)
            + struct.pack("<i", 48) + v1.tobytes() + struct.pack("<i", 48))
    assert raw == want
    t, npt, arrs, cex = checkpoint.read_particles_bak(path, 2)
    assert t == 1.5e-9 and npt.tolist() == [[2], [1]] and cex is None
    assert np.array_equal(arrs[0], v0) and np.array_equal(arrs[1], v1)


def test_subrecords_and_two_processes(tmp_path):
    """Records split into subrecords (gfortran: negative leading length =
    continues, negative trailing length = continuation), two OpenMP slices and
    the flag_cex records of tag_neg > 0."""
    rng = np.random.default_rng(3)
    npt = np.array([[5, 3], [0, 4]], dtype=np.int32)          # (ntype, nproc)
    arrs = [rng.standard_normal((int(npt[p, ip]), 6)) for ip in range(2) for p in range(2)]
    cex = [np.arange(int(npt[0, ip]), dtype=np.int32) for ip in range(2)]
    path = tmp_path / "p.bak"
    checkpoint.write_particles_bak(path, 2.0, npt, arrs, flag_cex=cex, max_sub=40)
    raw = path.read_bytes()
    # the first species record (5 x 48 = 240 bytes) at offset 16 + 24: subrecords of 40 bytes
    off = 16 + 24
    heads = []
    for k in range(6):
        h = struct.unpack_from("<i", raw, off)[0]
        t = struct.unpack_from("<i", raw, off + 4 + abs(h))[0]
        heads.append((h, t))
        off += 8 + abs(h)
    assert heads == [(-40, 40), (-40, -40), (-40, -40), (-40, -40), (-40, -40), (40, -40)]
    t, got_npt, got, got_cex = checkpoint.read_particles_bak(path, 2, nproc=2, tag_neg=1)
    assert np.array_equal(got_npt, npt)
    for a, b in zip(arrs, got):
        assert np.array_equal(a, b)
    for a, b in zip(cex, got_cex):
        assert np.array_equal(a, b)


def test_truncated_file_is_an_error(tmp_path):
    path = tmp_path / "p.bak"
    checkpoint.write_particles_bak(path, 0.0, [3], [np.zeros((3, 6))])
    path.write_bytes(path.read_bytes()[:-10])
    with pytest.raises(ValueError):
        checkpoint.read_particles_bak(path, 1)


@pytest.mark.gpu
@pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_save_and_restart_device_state(tmp_path, precision):
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("box16")
    a = Simulation(st, precision=precision, seed=5)
    a.load_uniform()
    for _ in range(3):
        a.step()
    path = tmp_path / "particles000.bak"
    a.save_bak(path, time=3 * st.dt)
    b = Simulation(st, precision=precision, seed=6)
    t = b.load_bak(path)
    assert t == 3 * st.dt
    assert np.array_equal(a.counts_host(), b.counts_host())
    for p in range(st.ntype):
        x, y = a.particles_f64(p).cpu().numpy(), b.particles_f64(p).cpu().numpy()
        tol = 0.0 if precision == "f64" else 1e-6
        assert np.abs(x - y).max() <= tol * np.abs(x).max()
    # the restart deposits the loaded particles with FP64 weights; the mixed
    # push deposits integer weights of 2^-20 (at most 5e-7 per weight apart)
    dtol = 1e-12 if precision == "f64" else 1e-5
    assert float((a.np - b.np).abs().max()) <= dtol * float(a.np.abs().max())
