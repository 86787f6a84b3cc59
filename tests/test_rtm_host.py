"""Host-side orchestration of ReverseTimeMigration (no GPU): the grid,
topography and snapshot-interval rules must land exactly where the reference
puts them (src/rtm.py:603-844), checked against the golden runs of the
reference source and against the interval figures of the workload configs."""
import numpy as np
import pytest

from oracle import fd_oracle
from taichirtm_b200.rtm import ReverseTimeMigration
from tests.conftest import load_golden


def _rtm_from(g):
    r = ReverseTimeMigration()
    r.set_observed_data(g["obs"][0], g["obs"][1], g["obs"][2])
    r.set_source(g["src_w"][0], g["src_w"][1], g["src_w"][2], float(g["src_x"]))
    r.set_receivers(g["rec_x"]).set_frequency(float(g["fs"])).set_boundary(int(g["fw"]))
    r.set_velocity_range(float(g["vmin"]), float(g["vmax"]), int(g["vstep"]))
    r.set_poisson_ratio(float(g["poisson"]))
    if g["heights"].size:
        r.set_topography(g["heights"])
    return r


@pytest.mark.parametrize("name", ["rtm_vfix", "rtm_vscan_topo"])
def test_grid_surface_and_locations_match_reference(name):
    g = load_golden(name)
    r = _rtm_from(g)
    v = float(g["v_fix"]) if np.isfinite(g["v_fix"]) else r.estimate_velocity(r.observed_v, r.vmin, r.vmax, r.vstep)
    dx, dz, nx, nz, rho, vs, vp = r._setup_modeling_conditions(v, float(g["cfl"]), int(g["fw"]))
    assert (nx, nz) == (int(g["nx"]), int(g["nz"]))
    assert dx == pytest.approx(float(g["dx"]), rel=1e-12)
    rec, src, sm = r._setup_surface_and_locations(nx, nz, dx, dz, int(g["fw"]))
    assert np.array_equal(np.asarray(src), g["src_loc_step"])
    if g["surface"].size:
        assert np.array_equal(r.surface_matrix, g["surface"])
    else:
        assert r.surface_matrix is None


def test_velocity_scan_matches_restatement():
    g = load_golden("rtm_vscan_topo")
    r = _rtm_from(g)
    v = r.estimate_velocity(r.observed_v, r.vmin, r.vmax, r.vstep)
    v_ref = fd_oracle.estimate_velocity(r.observed_v, r.receiver_loc, r.source_loc, r.fs, r.vmin, r.vmax, r.vstep)
    assert v == v_ref
    # the golden run's grid spacing encodes the velocity it picked: dx = v / fs / CFL
    assert v / float(g["fs"]) / float(g["cfl"]) == pytest.approx(float(g["dx"]), rel=1e-12)


@pytest.mark.parametrize("nx,nz,nt,nsrc,nrec,expect", [
    (301, 151, 2000, 1, 301, 1),     # plain P-SV workload
    (1001, 501, 4000, 1, 1001, 7),   # plain SH workload
    (2001, 801, 3000, 1, 600, 16),   # batched workload grid
    (1201, 401, 3000, 1, 1201, 5),   # FWI workload grid
])
def test_snapshot_interval_rule(nx, nz, nt, nsrc, nrec, expect):
    """_compute_isnap with the default 8 GB budget (rtm.py:719-844)."""
    assert ReverseTimeMigration()._compute_isnap(nx, nz, nt, nsrc, nrec) == expect


def test_check_parameters_messages():
    r = ReverseTimeMigration()
    with pytest.raises(ValueError, match="Observed data must be provided"):
        r.run()
    r.set_observed_data(np.zeros((2, 5)), np.zeros((2, 5)), np.zeros((2, 5)))
    with pytest.raises(ValueError, match="Source functions must be provided"):
        r.run()
    r.set_source(np.zeros(5), np.zeros(5), np.zeros(4), 1.0)
    r.set_receivers([0.0, 1.0]).set_frequency(100.0)
    with pytest.raises(ValueError, match="Source function shapes must match"):
        r.run()


def test_legacy_kwargs_constructor_warns():
    with pytest.warns(DeprecationWarning):
        r = ReverseTimeMigration(observed_u=np.zeros((2, 5)), observed_v=np.zeros((2, 5)),
                                 observed_w=np.zeros((2, 5)), source_u=np.zeros(5), source_v=np.zeros(5),
                                 source_w=np.zeros(5), receiver_loc=[0.0, 1.0], source_loc=0.5, fs=100.0)
    assert r.nt == 5 and r.absorbing_frame == 50 and r.isnap == 216


def _imaging_results(tmp_path):
    rng = np.random.default_rng(1)
    res = []
    for k in range(3):
        d = dict(u=rng.standard_normal((6, 4)).astype(np.float32), v=rng.standard_normal((6, 4)).astype(np.float32),
                 w=rng.standard_normal((6, 4)).astype(np.float32), offset=2.0, dx=0.5, dz=0.5, nx=6, nz=4)
        np.savez_compressed(tmp_path / f"s{k}.npz", **d)
        res.append(d)
    return res


def test_imaging_npz_load_and_save(tmp_path):
    from taichirtm_b200 import imaging
    res = _imaging_results(tmp_path)
    loaded = imaging.load_rtm_results(str(tmp_path))
    assert len(loaded) == 3 and all("filepath" in x for x in loaded)
    st = dict(u=res[0]["u"].T, v=res[0]["v"].T, w=res[0]["w"].T, xmin=-2.0, xmax=1.0, zmin=0.0, zmax=2.0)
    imaging.save_stacked_results(st, str(tmp_path / "out" / "stack.npz"))
    assert set(np.load(tmp_path / "out" / "stack.npz").files) == {"u", "v", "w", "xmin", "xmax", "zmin", "zmax"}


def test_imaging_stack_needs_a_gpu(tmp_path):
    """The cross-shot sum runs on the GPU in FP64; with no GPU visible it
    raises instead of summing on the host."""
    import torch

    from taichirtm_b200 import imaging
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError, match="CUDA"):
        imaging.stack_rtm_images(_imaging_results(tmp_path))


@pytest.mark.gpu
def test_imaging_stack_and_npz_roundtrip(tmp_path):
    from taichirtm_b200 import imaging
    res = _imaging_results(tmp_path)
    st = imaging.stack_rtm_images(res, subtract_mean=True)
    ref = sum(x["u"].astype(np.float64) for x in res).T
    ref = ref - ref.mean()
    assert np.allclose(st["u"], ref, atol=1e-5)
    assert st["extent"] == [-2.0, 1.0, 2.0, 0.0]
    imaging.save_stacked_results(st, str(tmp_path / "out" / "stack.npz"))
    assert set(np.load(tmp_path / "out" / "stack.npz").files) == {"u", "v", "w", "xmin", "xmax", "zmin", "zmax"}
