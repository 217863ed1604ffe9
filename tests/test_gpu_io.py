"""Restart files and BGEO particle output of the CUDA library
(SimulationBase::write / read, MpmSimulationBase::writeState / readState,
writePartio)."""
import struct

import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import build_scene

pytestmark = pytest.mark.gpu

DX = 1.0 / 64


def scene(precision="fp64", phase_field=False, plastic=False):
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, grid_log2=8)
    h, x = build_scene(s, kind="nh", n=6, dx=DX, seed=3, plastic=None)
    c = mpm.AnalyticCollisionObject(mpm.Sphere((0, 0, 0), 0.05), abi.SLIP, friction=0.1)
    c.setTranslation((0.45, 0.3, 0.45), (0.0, -0.5, 0.0))
    s.addCollisionObject(c)
    if phase_field:
        n = len(x)
        F = np.zeros((n, 3, 3))
        F[:, 0, 0] = 1 + 0.3 * (x[:, 0] - x[:, 0].min()) / np.ptp(x[:, 0])
        F[:, 1, 1] = F[:, 2, 2] = 1
        s.setParticles(F=F)
        h.addFBasedMpmForceWithPhaseField(0.05, 0.5 * DX)
        s.setPhaseFieldSolver(parabolic_M=1.0, cg_tolerance=1e-14)
    if plastic:
        h.addPlasticity(None, mpm.NonAssociativeCamClay(-0.01, 45.0, 0.3, 3.0, True))
    s.newton_tolerance = 1e-10
    s.newton_max_iterations = 8
    s.krylov_max_iterations = 80
    return s


def run(s, n, dt=1e-3):
    for _ in range(n):
        assert s.advanceOneTimeStep(dt) == abi.OK


@pytest.mark.parametrize("phase_field,plastic", [(False, False), (True, False), (False, True)])
def test_restart_continues_the_run(cuda_lib, tmp_path, phase_field, plastic):
    """A run restarted from a file written at step 3 ends where the run without
    the restart ends (FP64; the scatters' atomic order is the only difference)."""
    a = scene(phase_field=phase_field, plastic=plastic)
    run(a, 3)
    path = tmp_path / "restart_3.dat"
    a.write(path)
    run(a, 4)
    b = scene(phase_field=phase_field, plastic=plastic)
    b.read(path)
    assert abs(b.lib.time(b.ctx) - 3e-3) < 1e-15
    run(b, 4)
    pa, pb = a.getParticles(), b.getParticles()
    # the two runs differ only by the order of the atomic scatters, which the
    # Newton solve (tolerance 1e-10) carries into V and C
    for k, tol in (("X", 1e-10), ("F", 1e-8), ("V", 1e-6), ("C", 1e-5)):
        assert np.abs(pb[k] - pa[k]).max() <= tol * np.abs(pa[k]).max(), k
    if phase_field:
        np.testing.assert_allclose(b.getPhaseField()["c"], a.getPhaseField()["c"], rtol=0, atol=1e-9)
    if plastic:
        np.testing.assert_allclose(b.getLogJp(), a.getLogJp(), rtol=0, atol=1e-10)


def test_restart_rejects_mismatch_and_garbage(cuda_lib, tmp_path):
    a = scene()
    path = tmp_path / "r.dat"
    a.write(path)
    other = mpm.MpmSimulation(DX / 2, gravity=(0, -9.8, 0), grid_log2=8)
    with pytest.raises(abi.ZmpmError):
        other.read(path)
    bad = tmp_path / "bad.dat"
    bad.write_bytes(path.read_bytes()[:200])
    b = scene()
    x0 = b.getParticles()["X"].copy()
    with pytest.raises(abi.ZmpmError):
        b.read(bad)
    np.testing.assert_array_equal(b.getParticles()["X"], x0)  # a failed read leaves the scene


def test_restart_directory_layout(cuda_lib, tmp_path):
    """SimulationBase::write / read (SimulationBase.h:146-199): the state file
    restart_<frame>[_<substep>].dat beside last_written.txt and binary_ver.txt;
    a newer binary version is refused, a stale last frame warns."""
    a = scene()
    run(a, 2)
    out = tmp_path / "out"
    a.writeRestart(out, 2)
    a.writeRestart(out, 3, substep=4)
    assert sorted(p.name for p in out.iterdir()) == ["binary_ver.txt", "last_written.txt", "restart_2.dat", "restart_3_4.dat"]
    assert (out / "last_written.txt").read_text().strip() == "3"
    assert (out / "binary_ver.txt").read_text().strip() == str(abi.BINARY_VER)
    assert mpm.MpmSimulation.outputFileName(3, 4) == "restart_3_4.dat"
    assert mpm.MpmSimulation.outputFileName(2) == "restart_2.dat"
    b = scene()
    assert b.readRestart(out, 2) == 3
    for k in ("X", "V", "C", "F"):
        np.testing.assert_array_equal(b.getParticles()[k], a.getParticles()[k])
    # the last written frame (3) is before frame 5: stale data warns
    (out / "restart_5.dat").write_bytes((out / "restart_2.dat").read_bytes())
    with pytest.warns(UserWarning, match="stale"):
        b.readRestart(out, 5)
    # data of a newer binary version is refused, the scene kept
    (out / "binary_ver.txt").write_text(str(abi.BINARY_VER + 1))
    x0 = b.getParticles()["X"].copy()
    with pytest.raises(abi.ZmpmError, match="newer"):
        b.readRestart(out, 2)
    np.testing.assert_array_equal(b.getParticles()["X"], x0)
    # a missing version file reads as version 0 (accepted)
    (out / "binary_ver.txt").unlink()
    assert b.readRestart(out, 2) == 3


def read_bgeo(path):
    """Reader of the uncompressed BGEO v5 point files the library writes."""
    data = open(path, "rb").read()
    o = 0

    def take(fmt):
        nonlocal o
        v = struct.unpack_from(">" + fmt, data, o)
        o += struct.calcsize(">" + fmt)
        return v

    magic, = take("4s")
    vchar, = take("c")
    version, npts, nprims, npg, nprg, npa, nva, nprima, nattr = take("9i")
    assert (magic, vchar, version) == (b"Bgeo", b"V", 5)
    assert (nprims, npg, nprg, nva, nprima, nattr) == (0, 0, 0, 0, 0, 0)
    attrs = []
    for _ in range(npa):
        n, = take("H")
        name = data[o:o + n].decode()
        o += n
        size, typ = take("Hi")
        assert typ == 5
        take("%di" % size)
        attrs.append((name, size))
    width = 4 + sum(sz for _, sz in attrs)
    pts = np.frombuffer(data, dtype=">f4", count=npts * width, offset=o).reshape(npts, width)
    o += npts * width * 4
    assert data[o:] == b"\x00\xff"
    out = {"position": pts[:, :3], "w": pts[:, 3]}
    c = 4
    for name, sz in attrs:
        out[name] = pts[:, c:c + sz]
        c += sz
    return out


def test_bgeo_output(cuda_lib, tmp_path):
    s = scene(phase_field=True)
    run(s, 2)
    p = s.getParticles()
    s.writePartio(tmp_path / "partio_2.bgeo")
    g = read_bgeo(tmp_path / "partio_2.bgeo")
    assert set(g) == {"position", "w"}
    np.testing.assert_array_equal(g["position"], p["X"].astype(np.float32))
    np.testing.assert_array_equal(g["w"], 1.0)
    s.writePartio(tmp_path / "phaseField_2.bgeo", velocity=True, phase_field=True)
    g = read_bgeo(tmp_path / "phaseField_2.bgeo")
    np.testing.assert_array_equal(g["v"], p["V"].astype(np.float32))
    pf = s.getPhaseField()
    np.testing.assert_array_equal(g["pf"][:, 0], pf["c"].astype(np.float32))
    assert np.all(g["sigmaC"] > 0)


def test_restart_carries_admm_and_viscoelastic_state(cuda_lib, tmp_path):
    """ADMM multipliers, weights, last dv and the viscoelastic Fe travel in the
    restart file: the restarted ADMM run ends where the uninterrupted one ends."""
    def admm_scene():
        s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), grid_log2=8)
        h, x = build_scene(s, kind="hencky", n=6, dx=DX, seed=5, ground=0.1)
        E, nu = 1e4, 0.3
        nv = 2 * E / (2 * (1 + nu)) * 0.05
        h.addFElasticNonequilibratedBasedMpmForce(mpm.StvkWithHencky(E, nu), nv, nv)
        s.useAdmm(admm_max_iterations=10, rho_scale=0.8, global_tolerance=1e-12)
        return s
    a = admm_scene()
    run(a, 2, 2e-3)
    path = tmp_path / "admm.dat"
    a.write(path)
    run(a, 3, 2e-3)
    b = admm_scene()
    b.read(path)
    run(b, 3, 2e-3)
    pa, pb = a.getParticles(), b.getParticles()
    for k, tol in (("X", 1e-10), ("F", 1e-8), ("V", 1e-6)):
        assert np.abs(pb[k] - pa[k]).max() <= tol * np.abs(pa[k]).max(), k
    np.testing.assert_allclose(b.getViscoelasticStrain(), a.getViscoelasticStrain(), rtol=0, atol=1e-10)


def test_restart_explicit_run_is_reproduced(cuda_lib, tmp_path):
    a = scene()
    a.useExplicit()
    run(a, 5, 2e-4)
    path = tmp_path / "ex.dat"
    a.write(path)
    run(a, 5, 2e-4)
    b = scene()
    b.useExplicit()
    b.read(path)
    run(b, 5, 2e-4)
    pa, pb = a.getParticles(), b.getParticles()
    for k in ("X", "V", "F", "C"):
        assert np.abs(pb[k] - pa[k]).max() <= 1e-12 * max(np.abs(pa[k]).max(), 1.0), k
