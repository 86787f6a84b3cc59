"""Pins the oracle: the NumPy and C restatements against golden vectors recorded
from the unmodified reference source (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle import c_oracle, fd_oracle
from tests.conftest import load_golden, rel_l2, same_with_nan

FWBW = ["fwbw_basic", "fwbw_topo", "fwbw_narrow", "fwbw_edge_source"]


def _args(g):
    return dict(dx=float(g["dx"]), dz=float(g["dz"]), nt=int(g["nt"]), fs=float(g["fs"]),
                fw=int(g["fw"]))


def _surface(g):
    return g["surface"] if g["surface"].size else None


@pytest.mark.parametrize("name", FWBW)
def test_numpy_oracle_bit_exact_vs_reference(name):
    """FP64 NumPy restatement == reference source run in FP64, bit for bit."""
    g = load_golden(name)
    sm, a = _surface(g), _args(g)
    assert np.array_equal(fd_oracle.sponge(int(g["nx"]), int(g["nz"]), int(g["fw"])), g["absorb"])
    m = fd_oracle.derived_material(g["mu_s"], g["lam_s"], g["rho_s"])
    for k in ("mxz", "myx", "myz", "inv_rho", "inv_rho_u", "inv_rho_w"):
        assert np.array_equal(m[k], g[k]), k
    kw = dict(src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"], rec=g["rec"],
              isnap=int(g["isnap"]), surface=sm, check_interval=0, **a)
    obs = fd_oracle.forward(g["mu_t"], g["lam_t"], g["rho_t"], **kw)
    syn = fd_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], save=True, **kw)
    img = fd_oracle.backward(g["mu_s"], g["lam_s"], g["rho_s"], rec=g["rec"], ou=g["obs"][0],
                             ov=g["obs"][1], ow=g["obs"][2], snaps=syn["snaps"],
                             isnaps=syn["isnaps"], num_snaps=syn["num_snaps"],
                             isnap=int(g["isnap"]), surface=sm, check_interval=0, **a)
    assert np.array_equal(obs["seis"], g["obs"], equal_nan=True)
    assert np.array_equal(syn["seis"], g["syn"], equal_nan=True)
    if name != "fwbw_edge_source":
        assert np.array_equal(syn["snaps"], g["snaps"], equal_nan=True)
        assert np.array_equal(syn["isnaps"], g["isnaps"])
        assert np.array_equal(img["img"], g["img"], equal_nan=True)


@pytest.mark.parametrize("name", FWBW)
def test_c_oracle_f64_vs_reference(name):
    g = load_golden(name)
    sm, a = _surface(g), _args(g)
    kw = dict(src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"], rec=g["rec"],
              isnap=int(g["isnap"]), surface=sm, check_interval=0, dtype=np.float64, **a)
    f = c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], save=True, **kw)
    assert same_with_nan(f["seis"], g["syn"], rtol=1e-12, atol=1e-12 * np.nanmax(np.abs(g["syn"][np.isfinite(g["syn"])])))
    snaps_ref_layout = np.moveaxis(f["snaps"], 1, -1)
    b = c_oracle.backward(g["mu_s"], g["lam_s"], g["rho_s"], rec=g["rec"], obs=g["obs"],
                          snaps=f["snaps"], isnaps=f["isnaps"], num_snaps=f["num_snaps"],
                          isnap=int(g["isnap"]), surface=sm, check_interval=0,
                          dtype=np.float64, **a)
    if name != "fwbw_edge_source":
        assert same_with_nan(snaps_ref_layout, g["snaps"], atol=1e-12 * np.abs(g["snaps"]).max())
        assert rel_l2(b["img"], g["img"]) < 1e-12


def test_edge_source_failure_code():
    """A source on an edge cell multiplies by inv_rho_u = 1/0 (fm:304-307): the
    first finite check (it = 0) reports code 3 (w beats u, fm:471-472)."""
    g = load_golden("fwbw_edge_source")
    a = _args(g)
    kw = dict(src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"], rec=g["rec"], isnap=2, **a)
    assert fd_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], **kw)["flag"] == 3
    assert c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], dtype=np.float64, **kw)["flag"] == 3
    assert c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], dtype=np.float32, **kw)["flag"] == 3


def test_reference_f32_harmonic_mean_overflows():
    """The reference's f32 4-point harmonic mean (fm:271-276) multiplies four
    moduli; for mu ~ 1e10 Pa (Vp 3500 m/s rock) the product overflows f32 and
    the run goes non-finite at the first check.  The FP64 set-up avoids it."""
    nx, nz, nt = 24, 20, 12
    mu = np.full((nx, nz), 1.0e10, np.float32)
    lam = np.full((nx, nz), 1.2e10, np.float32)
    rho = np.full((nx, nz), 2400.0, np.float32)
    w = np.zeros((1, nt), np.float32)
    w[0, 1] = 1.0
    kw = dict(dx=5.0, dz=5.0, nt=nt, fs=2000.0, fw=4, src=[[12, 5]], wu=w, wv=w, ww=w,
              rec=[[12, 1]], check_interval=1, dtype=np.float32)
    assert c_oracle.forward(mu, lam, rho, setup_f64=False, **kw)["flag"] != 0
    assert c_oracle.forward(mu, lam, rho, setup_f64=True, **kw)["flag"] == 0
    m32 = fd_oracle.derived_material(mu, lam, rho, np.float32)
    assert np.isinf(m32["mxz"][1:-1, 1:-1]).all()


def test_c_f32_close_to_f64():
    g = load_golden("fwbw_basic")
    a = _args(g)
    kw = dict(src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"], rec=g["rec"], **a)
    f64 = c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], dtype=np.float64, **kw)
    f32 = c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], dtype=np.float32, **kw)
    assert rel_l2(f32["seis"], f64["seis"]) < 1e-5


def test_modes_split_exact():
    """P-SV and SH never read each other's fields (fm:330-384): running one
    mode alone gives the same numbers for its components."""
    g = load_golden("fwbw_basic")
    a = _args(g)
    kw = dict(src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"], rec=g["rec"], dtype=np.float64, **a)
    both = c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], modes=3, **kw)["seis"]
    psv = c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], modes=1, **kw)["seis"]
    sh = c_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], modes=2, **kw)["seis"]
    assert np.array_equal(both[[0, 2]], psv[[0, 2]])
    assert np.array_equal(both[1], sh[1])


def test_imaging_slots_and_source_normalization_definition():
    """The imaging-step gate restated for the source-normalised condition
    selects exactly the slots the golden backward runs correlate, and the
    normalisation divides by sum snapshot^2 + eps * max (0 where that is 0)."""
    g = load_golden("fwbw_basic")
    nt, isnap, ns = int(g["nt"]), int(g["isnap"]), int(g["num_snaps"])
    slots = fd_oracle.imaging_slots(nt, isnap, g["isnaps"], ns)
    ts = [(nt - 1) - it for it in range(nt)]
    want = [t // isnap - 1 for t in ts if t > 0 and t % isnap == 0 and t // isnap - 1 < ns
            and int(g["isnaps"][t // isnap - 1]) == t]
    assert slots == want and len(slots) > 0
    rng = np.random.default_rng(3)
    snaps = rng.standard_normal((3, 5, 4, 6))
    snaps[1] = 0.0
    img = rng.standard_normal((3, 5, 4))
    out = fd_oracle.source_normalized(img, snaps, [0, 2, 5], 0.1)
    ill = (snaps[0][..., [0, 2, 5]] ** 2).sum(-1)
    assert np.allclose(out[0], img[0] / (ill + 0.1 * ill.max()))
    assert np.all(out[1] == 0.0)


def test_c_oracle_snapshot_components_subset_images_the_same():
    """Keeping only the imaged components' snapshots (snap_comps) gives the
    same image for those components and zero for the others."""
    from oracle import c_oracle
    from taichirtm_b200 import synthetic as S
    s = S.config1(nt=120)
    sh = s.shots[0]
    mu, lam, rho = s.material()
    kw = dict(dx=s.dx, dz=s.dz, nt=s.nt, fs=s.fs, fw=s.fw, dtype=np.float64, modes=1)
    wv = dict(wu=sh.wavelets[0], wv=sh.wavelets[1], ww=sh.wavelets[2])
    f3 = c_oracle.forward(mu, lam, rho, src=sh.src, rec=sh.rec, save=True, isnap=3, **wv, **kw)
    f2 = c_oracle.forward(mu, lam, rho, src=sh.src, rec=sh.rec, save=True, isnap=3, snap_comps=(0, 2), **wv, **kw)
    assert f2["snaps"].shape[0] == 2
    obs = 0.5 * f3["seis"]
    b3 = c_oracle.backward(mu, lam, rho, rec=sh.rec, obs=obs, snaps=f3["snaps"], isnaps=f3["isnaps"],
                           num_snaps=f3["num_snaps"], isnap=3, **kw)
    b2 = c_oracle.backward(mu, lam, rho, rec=sh.rec, obs=obs, snaps=f2["snaps"], isnaps=f2["isnaps"],
                           num_snaps=f2["num_snaps"], isnap=3, snap_comps=(0, 2), **kw)
    assert np.array_equal(b3["img"][[0, 2]], b2["img"][[0, 2]])
    assert np.abs(b2["img"][1]).max() == 0.0
