"""The ctypes binding a TaichiRTM maintainer would add
(taichirtm_b200/reference_binding.py), loaded on the in-tree library and run
against the package's own ForwardModeling: the same seismograms and status
code."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_integration_stub_matches_forward_modeling():
    from taichirtm_b200 import ForwardModeling, _lib, reference_binding
    lib = reference_binding.load(_lib.lib()._name)  # the in-tree librtm_b200.so the package loads
    nx, nz, nt, fw = 60, 48, 120, 10
    rng = np.random.default_rng(2)
    vp = 2200.0 + 300.0 * rng.random((nx, nz))
    vs, rho = vp / 1.8, 310.0 * vp ** 0.25
    mu = (rho * vs ** 2).astype(np.float32)
    lam = (rho * vp ** 2 - 2 * rho * vs ** 2).astype(np.float32)
    rho = rho.astype(np.float32)
    src = np.array([[30, 3]], np.int32)
    rec = np.array([[i, 1] for i in range(nx)], np.int32)
    t = np.arange(nt) / 2000.0 - 0.02
    a = (np.pi * 40.0 * t) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    wav = np.stack([0.3 * w, 0.5 * w, w])[:, None, :]
    dev = torch.device("cuda")
    d = {k: torch.as_tensor(v, device=dev).contiguous() for k, v in dict(mu=mu, lam=lam, rho=rho, wav=wav).items()}
    seis = torch.zeros((3, len(rec), nt), dtype=torch.float32, device=dev)
    flag = reference_binding.run_forward(lib, nx, nz, 5.0, 5.0, nt, 2000.0, fw, d["mu"], d["lam"], d["rho"], src, rec, d["wav"], seis,
                             stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    fo = ForwardModeling(nx=nx, nz=nz, dx=5.0, dz=5.0, nt=nt, fs=2000.0, absorbing_frame=fw, mu_field=mu,
                         lam_field=lam, rho_field=rho, src_loc_field=src, wavelet_u_field=wav[0],
                         wavelet_v_field=wav[1], wavelet_w_field=wav[2], recv_loc_field=rec, num_sources=1,
                         num_receivers=len(rec))
    assert fo.run() == flag == 0
    ref = np.stack(fo.get_seismogram())
    assert np.abs(ref).max() > 0
    assert np.array_equal(seis.cpu().numpy(), ref)
