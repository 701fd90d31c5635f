"""The reference's on-disk formats (germaine_b200.files over gm_write_seis,
gm_read_seis, gm_write_model_true, gm_write_model, gm_read_model): files
written here are byte-identical to the ones write_seis_AC
(src/AC/write_seis_AC.c:53-67), writemod_true (src/writemod_true.c:26-34)
and writemod (src/writemod.c:24-30) write, and reading a file gives what
read_seis_AC (src/AC/read_seis_AC.c:24-37) and readmod
(src/readmod.c:43-104) give.  Pinned against the reference's bytes in
tests/golden/files_formats.npz, against the oracle's restatement, and (where
oracle/_ref is built) against the reference run live.  Host code only."""
import os

import numpy as np
import pytest

import oracle as O
from germaine_b200 import GmError, files
from tests.test_oracle_pin import GOLDEN, _bits

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference tree absent)")


def _cases():
    d = np.load(os.path.join(GOLDEN, "files_formats.npz"))
    for k in range(int(d["ngrids"])):
        nx, ny, npml, fs = (int(v) for v in d[f"case_{k}"])
        sfx = f"_{k}"
        yield O.Grid(nx=nx, ny=ny, dh=10.0, npml=npml, free_surf=fs), {
            key[:-len(sfx)]: d[key] for key in d.files if key.endswith(sfx)}


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def test_reference_zeroes_last_seismogram_sample():
    """write_seis_AC's gather misses element n: the fixture's file holds the
    input except its last complex sample, which is 0."""
    for _, c in _cases():
        got = c["seis_file"].view(np.complex64)
        want = c["seis"].reshape(-1)
        assert np.array_equal(got[:-1].view(np.float32), want[:-1].view(np.float32))
        assert got[-1] == 0 and want[-1] != 0


def test_oracle_restatement_against_reference_bytes():
    for g, c in _cases():
        p = O.Port(g)
        assert p.seis_bytes(c["seis"]) == c["seis_file"].tobytes()
        assert p.model_true_bytes(c["grid"]) == c["true_file"].tobytes()
        assert p.model_true_bytes(c["grid"], 2, 3) == c["true2_file"].tobytes()
        assert p.model_bytes(c["grid"]) == c["full_file"].tobytes()
        for name in ("vp", "rho"):
            got = p.model_from_bytes(c[name].tobytes())
            assert np.array_equal(_bits(got), _bits(c["readmod_" + name]))


def test_writers_match_reference_bytes(tmp_path):
    for g, c in _cases():
        sp = files.seis_path(str(tmp_path / "picks"), 2)
        files.write_seis(sp, c["seis"])
        assert _read(sp) == c["seis_file"].tobytes()
        files.write_seis(tmp_path / "all.bin", c["seis"], keep_last=True)
        assert _read(tmp_path / "all.bin") == O.Port(g).seis_bytes(c["seis"], keep_last=True)
        files.write_model_true(tmp_path / "t1", c["grid"], g.npml, g.free_surf)
        assert _read(tmp_path / "t1") == c["true_file"].tobytes()
        files.write_model_true(tmp_path / "t2", c["grid"], g.npml, g.free_surf, idx=2, idy=3)
        assert _read(tmp_path / "t2") == c["true2_file"].tobytes()
        files.write_model(tmp_path / "f1", c["grid"])
        assert _read(tmp_path / "f1") == c["full_file"].tobytes()


def test_readers_match_reference(tmp_path):
    for g, c in _cases():
        sp = tmp_path / "obs_p_stage_2.bin"
        sp.write_bytes(c["seis_file"].tobytes())
        got = files.read_seis(sp, *c["seis"].shape)
        assert got.tobytes() == c["seis_file"].tobytes()
        for name in ("vp", "rho"):
            mp = tmp_path / f"m.{name}"
            mp.write_bytes(c[name].tobytes())
            got = files.read_model(mp, g.nx, g.ny, g.npml, g.free_surf)
            assert np.array_equal(_bits(got), _bits(c["readmod_" + name]))


def test_round_trips(tmp_path):
    """writemod_true then readmod gives back a model already extended into
    the frame; seismograms written with keep_last read back unchanged."""
    rng = np.random.default_rng(4)
    for nx, ny, npml, fs in [(40, 30, 6, 0), (40, 30, 6, 1), (17, 9, 0, 0)]:
        g = O.Grid(nx=nx, ny=ny, dh=5.0, npml=npml, free_surf=fs)
        inner = rng.standard_normal((ny - npml - g.fsshift, nx - 2 * npml)).astype(np.float32)
        full = np.pad(inner, ((g.fsshift, npml), (npml, npml)), mode="edge")
        files.write_model_true(tmp_path / "m", full, npml, fs)
        back = files.read_model(tmp_path / "m", nx, ny, npml, fs)
        assert np.array_equal(_bits(back), _bits(full))
    seis = (rng.standard_normal((2, 5, 7)) + 1j * rng.standard_normal((2, 5, 7))).astype(np.complex64)
    files.write_seis(tmp_path / "s.bin", seis, keep_last=True)
    assert np.array_equal(files.read_seis(tmp_path / "s.bin", 2, 5, 7).view(np.float32), seis.view(np.float32))


def test_errors(tmp_path):
    with pytest.raises(GmError):
        files.read_seis(tmp_path / "missing.bin", 1, 1, 1)
    (tmp_path / "short.bin").write_bytes(b"\0" * 12)
    with pytest.raises(GmError):
        files.read_seis(tmp_path / "short.bin", 1, 1, 2)
    with pytest.raises(GmError):
        files.read_model(tmp_path / "short.bin", 10, 10, 2, 0)
    with pytest.raises(GmError):   # no interior
        files.write_model_true(tmp_path / "x", np.zeros((4, 4), np.float32), 2, 0)
    with pytest.raises(GmError):
        files.write_model(tmp_path / "x", np.zeros((4, 4), np.float32), idx=0)
    with pytest.raises(GmError):
        files.write_seis(tmp_path / "no_such_dir" / "s.bin", np.zeros((1, 1, 1), np.complex64))


@needs_ref
def test_against_reference_live(short_tmp):
    """Fresh seeded data through the reference's own writers and readers."""
    import pathlib
    tmp_path = pathlib.Path(short_tmp)
    rng = np.random.default_rng(31)
    for nx, ny, npml, fs in [(33, 25, 7, 0), (25, 20, 3, 1)]:
        g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=npml, free_surf=fs)
        ref = O.Ref(g)
        seis = (rng.standard_normal((2, 3, 11)) + 1j * rng.standard_normal((2, 3, 11))).astype(np.complex64)
        ref.write_seis(str(tmp_path / "r"), 5, seis)
        files.write_seis(files.seis_path(str(tmp_path / "o"), 5), seis)
        assert _read(tmp_path / "r_p_stage_5.bin") == _read(tmp_path / "o_p_stage_5.bin")
        back = ref.read_seis(str(tmp_path / "o"), 5, 2, 3, 11)
        assert back.tobytes() == files.read_seis(tmp_path / "o_p_stage_5.bin", 2, 3, 11).tobytes()
        grid = rng.standard_normal((ny, nx)).astype(np.float32)
        for idx, idy in [(1, 1), (3, 2)]:
            ref.writemod_true(str(tmp_path / "rt"), grid, idx, idy)
            files.write_model_true(tmp_path / "ot", grid, npml, fs, idx=idx, idy=idy)
            assert _read(tmp_path / "rt") == _read(tmp_path / "ot")
            ref.writemod(str(tmp_path / "rf"), grid, idx, idy)
            files.write_model(tmp_path / "of", grid, idx=idx, idy=idy)
            assert _read(tmp_path / "rf") == _read(tmp_path / "of")
        files.write_model_true(tmp_path / "mm.vp", grid, npml, fs)
        files.write_model_true(tmp_path / "mm.rho", grid * 2, npml, fs)
        rvp, rrho = ref.readmod(str(tmp_path / "mm"))
        assert np.array_equal(_bits(rvp), _bits(files.read_model(tmp_path / "mm.vp", nx, ny, npml, fs)))
        assert np.array_equal(_bits(rrho), _bits(files.read_model(tmp_path / "mm.rho", nx, ny, npml, fs)))
        # readmod's own copy of the extended model (writemod format 3)
        files.write_model(tmp_path / "ours.vp", rvp)
        assert _read(tmp_path / "mm.germaine.vp") == _read(tmp_path / "ours.vp")


def test_read_grid_round_trip(tmp_path):
    rng = np.random.default_rng(12)
    grid = rng.standard_normal((23, 31)).astype(np.float32)
    files.write_model(tmp_path / "g", grid)
    assert np.array_equal(_bits(files.read_grid(tmp_path / "g", 31, 23)), _bits(grid))
    with pytest.raises(GmError):
        files.read_grid(tmp_path / "g", 31, 24)   # file too short


@needs_ref
def test_read_grid_of_reference_lbfgs_files(short_tmp):
    """The reference's l-BFGS state files (src/LBFGS.c:183-216) read back as
    the grids it was given and returned."""
    from tests import lbfgs_cases as LC
    g = LC.grid()
    (gr, gm, md, _), = LC.sequence(g, 1, 1, seed=13)
    jac = os.path.join(short_tmp, "j")
    ref = O.RefLbfgs(g, 2, 1, jac)
    hgrad = ref.step_ac(1, 1, gr, gm, md)
    assert np.array_equal(_bits(files.read_grid(jac + "_p.old", g.nx, g.ny)), _bits(gr))
    assert np.array_equal(_bits(files.read_grid(jac + "_p_vp.old", g.nx, g.ny)), _bits(md))
    assert np.array_equal(_bits(files.read_grid(jac + "_c.old", g.nx, g.ny)), _bits(hgrad))
