"""display_callback through the reference-shaped classes: the sequence of
(step, u, v, w) the callback receives equals the reference loop's
(forward_modeling.py:553-559: every it % isnap == 0, it = 0 included, the
live wavefield before that step's finite check; backward_modeling.py:565-569:
every imaging step t, the backward wavefield after its correlation), bit for
bit against the NumPy FP32 restatement of those loops, for one and two
steps per launch; after a failed finite check no callback follows; an
exception raised by the callback stops the run and propagates."""
import numpy as np
import pytest

from oracle import fd_oracle
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu

SHAPES = [None, dict(vec=2, rows=8, warps=2, tsteps=2, prefetch=3), dict(vec=4, rows=5, warps=1, tsteps=2)]


def _kwargs(g, tune):
    nx, nz, nt = int(g["nx"]), int(g["nz"]), int(g["nt"])
    return dict(nx=nx, nz=nz, dx=float(g["dx"]), dz=float(g["dz"]), nt=nt, fs=float(g["fs"]),
                absorbing_frame=int(g["fw"]), src_loc_field=g["src"], recv_loc_field=g["rec"],
                num_sources=len(g["src"]), num_receivers=len(g["rec"]), mu_field=g["mu_s"], lam_field=g["lam_s"],
                rho_field=g["rho_s"], tune=tune)


def _same(a, b):
    assert [x[0] for x in a] == [x[0] for x in b]
    for x, y in zip(a, b):
        for c in range(1, 4):
            assert np.array_equal(np.asarray(x[c]), np.asarray(y[c]), equal_nan=True), (x[0], c)


@pytest.mark.parametrize("tune", SHAPES)
def test_display_callback_sequences_equal_the_reference_loops(tune):
    from taichirtm_b200 import BackwardModeling, ForwardModeling
    g = load_golden("fwbw_basic")
    isnap = int(g["isnap"])
    kw = dict(dx=float(g["dx"]), dz=float(g["dz"]), nt=int(g["nt"]), fs=float(g["fs"]), fw=int(g["fw"]))
    ref_f, ref_b, got_f, got_b = [], [], [], []
    ref = fd_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"],
                            rec=g["rec"], isnap=isnap, save=True, dtype=np.float32, setup_f64=True,
                            display_callback=lambda u, v, w, it: ref_f.append((it, u, v, w)), **kw)
    fd_oracle.backward(g["mu_s"], g["lam_s"], g["rho_s"], rec=g["rec"], ou=g["obs"][0], ov=g["obs"][1],
                       ow=g["obs"][2], snaps=ref["snaps"], isnaps=ref["isnaps"], num_snaps=ref["num_snaps"],
                       isnap=isnap, dtype=np.float32, setup_f64=True, kahan=True,
                       display_callback=lambda u, v, w, t: ref_b.append((t, u, v, w)), **kw)
    a = _kwargs(g, tune)
    fo = ForwardModeling(isnap=isnap, wavelet_u_field=g["wu"], wavelet_v_field=g["wv"], wavelet_w_field=g["ww"], **a)
    assert fo.run(save=True, display_callback=lambda u, v, w, it, nx, nz, dx, dz: got_f.append((it, u, v, w))) == 0
    assert got_f[0][0] == 0 and len(got_f) == (int(g["nt"]) - 1) // isnap + 1
    _same(got_f, ref_f)
    bw = BackwardModeling(obsdata_u_field=g["obs"][0], obsdata_v_field=g["obs"][1], obsdata_w_field=g["obs"][2], **a)
    assert bw.run_calc(fo.u_save_field, fo.v_save_field, fo.w_save_field, fo.isnaps_field, fo.num_snaps, isnap,
                       display_callback=lambda u, v, w, t, nx, nz, dx, dz: got_b.append((t, u, v, w))) == 0
    assert len(got_b) == len(ref_b) > 0
    _same(got_b, ref_b)
    # the run without a callback gives the same results
    fo2 = ForwardModeling(isnap=isnap, wavelet_u_field=g["wu"], wavelet_v_field=g["wv"], wavelet_w_field=g["ww"], **a)
    assert fo2.run(save=True) == 0
    assert np.array_equal(np.stack(fo2.get_seismogram()), np.stack(fo.get_seismogram()))
    for x in (fo, fo2, bw):
        x.cleanup()


def test_no_display_callback_after_a_failed_check():
    """A source on an edge cell injects inf (code 3, forward_modeling.py:437-443):
    callbacks up to and including the failing check step, none after."""
    from taichirtm_b200 import ForwardModeling
    g = load_golden("fwbw_edge_source")
    isnap = 2
    kw = dict(dx=float(g["dx"]), dz=float(g["dz"]), nt=int(g["nt"]), fs=float(g["fs"]), fw=int(g["fw"]))
    ref_f, got_f = [], []
    with np.errstate(all="ignore"):
        ref = fd_oracle.forward(g["mu_s"], g["lam_s"], g["rho_s"], src=g["src"], wu=g["wu"], wv=g["wv"], ww=g["ww"],
                                rec=g["rec"], isnap=isnap, check_interval=3, dtype=np.float32, setup_f64=True,
                                display_callback=lambda u, v, w, it: ref_f.append((it, u, v, w)), **kw)
    assert ref["flag"] > 0
    for tune in SHAPES:
        got_f.clear()
        fo = ForwardModeling(isnap=isnap, wavelet_u_field=g["wu"], wavelet_v_field=g["wv"], wavelet_w_field=g["ww"],
                             **_kwargs(g, tune))
        code = fo.run(stability_check_interval=3,
                      display_callback=lambda u, v, w, it, nx, nz, dx, dz: got_f.append((it, u, v, w)))
        assert code == ref["flag"]
        _same(got_f, ref_f)
        fo.cleanup()


def test_display_callback_exception_propagates():
    from taichirtm_b200 import ForwardModeling
    g = load_golden("fwbw_basic")
    fo = ForwardModeling(isnap=int(g["isnap"]), wavelet_u_field=g["wu"], wavelet_v_field=g["wv"],
                         wavelet_w_field=g["ww"], **_kwargs(g, None))
    seen = []

    def cb(u, v, w, it, nx, nz, dx, dz):
        seen.append(it)
        if len(seen) == 2:
            raise KeyError("stop here")
    with pytest.raises(KeyError, match="stop here"):
        fo.run(display_callback=cb)
    assert len(seen) == 2
    assert fo.run() == 0  # the plan is usable afterwards
    fo.cleanup()
