"""glb_lens_rayshoot_noalloc, the entry point for callers that cannot allocate
device memory while they shoot rays (cudaMalloc / cudaFree synchronise the
device and may fail under a memory cap): its results must equal those of
glb_lens_rayshoot_device on the same lens and rays, on two calls in a row
(the calls share one fixed scratch array).  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import slsimlib_b200 as glb
from slsimlib_b200 import synth

pytestmark = pytest.mark.gpu


def _lens():
    spec = synth.light_cone(seed=51, n_total=40000, n_planes=3, halos_per_plane=4)
    spec.halos.append(synth.NFWHalo(3e13, 0.4, 0.7, 6.0))
    L = glb.Lens(spec.zsource)
    for h in spec.halos:
        if isinstance(h, synth.ParticlePlane):
            L.insertMainHalo(glb.LensHaloParticles(h.particles, h.z), True)
        elif isinstance(h, synth.NSIEHalo):
            L.insertMainHalo(glb.LensHaloRealNSIE(h.mass, h.z, h.sigma, h.rcore, h.fratio, h.pa), True)
        else:
            L.insertMainHalo(glb.LensHaloNFW(h.mass, h.rsize, h.z, h.conc), True)
    return L


def _rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("precision", [glb.PREC_FP64, glb.PREC_SPLIT])
def test_noalloc_matches_allocating_entry_point(precision):
    import torch
    L = _lens()
    lib = glb.load_library()
    rng = np.random.default_rng(7)
    dev = torch.device("cuda", 0)
    for call in range(2):  # two calls in a row through the shared scratch
        n = 40000 if call == 0 else 12345
        x = torch.from_numpy(rng.uniform(-30, 30, (n, 2)) * synth.ARCSEC).to(dev)
        zs = torch.from_numpy(rng.uniform(0.3, 3.0, n)).to(dev) if call == 1 else None
        zp = zs.data_ptr() if zs is not None else None
        y_ref = torch.empty((n, 2), dtype=torch.float64, device=dev)
        A_ref = torch.empty((n, 4), dtype=torch.float64, device=dev)
        y = torch.full((n, 2), np.nan, dtype=torch.float64, device=dev)
        A = torch.full((n, 4), np.nan, dtype=torch.float64, device=dev)
        s = torch.cuda.current_stream().cuda_stream or None
        torch.cuda.synchronize()  # the tensors above were filled on torch's stream
        glb._check(lib.glb_lens_rayshoot_device(L._h, n, x.data_ptr(), zp, y_ref.data_ptr(), A_ref.data_ptr(),
                                                precision, s))
        torch.cuda.synchronize()
        glb._check(lib.glb_lens_rayshoot_noalloc(L._h, n, x.data_ptr(), zp, y.data_ptr(), A.data_ptr(),
                                                 precision, s))
        torch.cuda.synchronize()
        y_ref, A_ref, y, A = (t.cpu().numpy() for t in (y_ref, A_ref, y, A))
        assert np.all(np.isfinite(y)) and np.all(np.isfinite(A))
        assert _rel(y, y_ref) < 1e-9
        assert np.max(np.abs(A - A_ref)) < 1e-9


def test_noalloc_rejects_oversized_calls():
    L = _lens()
    lib = glb.load_library()
    rc = lib.glb_lens_rayshoot_noalloc(L._h, 65537, C.c_void_p(1), None, C.c_void_p(1), C.c_void_p(1), 0, None)
    assert rc == glb.GLB_ERR_ARG
    assert b"65536" in lib.glb_last_error()
