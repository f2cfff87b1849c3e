"""The allocation-free demag entry point against the regular entry point.

fullmag_fdm_demag_field_f64_noalloc exists for callers that cannot let this
library allocate device memory (a host framework owning the whole device
budget, or a loop that must not pay cudaMalloc's implicit synchronisation).
It keeps its FFT work arrays in a fixed 32 MiB device array instead.  Here it
is called through the C ABI twice in a row, on two different magnetisations,
and each result is compared with H_demag from fullmag_fdm_backend_create +
refresh_observables, within the FP64 field tolerance of the other parity
tests (1e-13 relative to max |H|).  The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf

pytestmark = pytest.mark.gpu


def _entry():
    lib = nf.load_library()
    fn = lib.fullmag_fdm_demag_field_f64_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p,
                   C.c_double, C.c_void_p, C.c_void_p, C.c_char_p, C.c_uint64]
    return fn


def _octant(spectra, nx, ny, nz, thin):
    """Real octant [6][KZ][nx+1][ny+1] of the interleaved host spectra."""
    Lx, Ly, Lz = 2 * nx, 2 * ny, (1 if thin else 2 * nz)
    KZ = 1 if thin else nz + 1
    out = []
    for s in spectra:
        re = s[0::2].reshape(Lz, Ly, Lx)
        out.append(re[:KZ, :ny + 1, :nx + 1].transpose(0, 2, 1))
    return np.ascontiguousarray(np.stack(out))


# nz = 1 thin (2-D y pass), and 3-D with 2nz = 2, 4, 8 and 16 (the z FFT pass at each length)
@pytest.mark.parametrize("cells,thin", [((64, 32, 1), True), ((16, 16, 1), False), ((32, 16, 2), False),
                                        ((32, 16, 4), False), ((16, 8, 8), False)])
def test_noalloc_demag_matches_regular_entry_point(cells, thin):
    import torch

    nx, ny, nz = cells
    n = nx * ny * nz
    d = (2e-9, 2.5e-9, 3e-9)
    ms = 8.0e5
    spectra = nf.newell_spectra(nx, ny, nz, *d, thin_film_2d=thin)
    m_a = nf.random_unit_vectors(11, n)
    m_b = nf.random_unit_vectors(12, n)
    plan = nf.FdmPlan(cells=cells, cell_size=d, initial_magnetization=m_a, saturation_magnetisation=ms,
                      enable_exchange=False, demag_spectra=spectra)
    be = nf.NativeFdmBackend(plan)
    ref_a = be.copy_field(nf.OBS_H_DEMAG)
    be.upload_m(m_b)
    be.refresh_observables()
    ref_b = be.copy_field(nf.OBS_H_DEMAG)
    be.close()

    fn = _entry()
    dev = torch.device("cuda", 0)
    octant = torch.from_numpy(_octant(spectra, nx, ny, nz, thin)).to(dev)
    h = torch.empty(3 * n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    err = C.create_string_buffer(512)
    for m_aos, ref in ((m_a, ref_a), (m_b, ref_b)):
        m_soa = torch.from_numpy(np.ascontiguousarray(m_aos.reshape(n, 3).T)).to(dev)
        h.fill_(float("nan"))
        rc = fn(nx, ny, nz, int(thin), octant.data_ptr(), m_soa.data_ptr(), ms, h.data_ptr(),
                stream, err, len(err))
        assert rc == nf.OK, err.value.decode()
        torch.cuda.synchronize()
        got = h.cpu().numpy().reshape(3, n).T.reshape(-1)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-13 * scale


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    fn = _entry()
    err = C.create_string_buffer(512)
    dev = torch.device("cuda", 0)
    dummy = torch.zeros(16, dtype=torch.float64, device=dev)
    rc = fn(512, 512, 8, 0, dummy.data_ptr(), dummy.data_ptr(), 8e5, dummy.data_ptr(), None,
            err, len(err))
    assert rc == nf.ERR_INVALID
    assert b"at most" in err.value and b"bytes" in err.value
    rc = fn(12, 8, 1, 1, dummy.data_ptr(), dummy.data_ptr(), 8e5, dummy.data_ptr(), None,
            err, len(err))
    assert rc == nf.ERR_INVALID and b"powers of two" in err.value
    # sizes far beyond the limits are rejected before any length is formed
    rc = fn(0x80000000, 8, 1, 1, dummy.data_ptr(), dummy.data_ptr(), 8e5, dummy.data_ptr(), None,
            err, len(err))
    assert rc == nf.ERR_INVALID and b"powers of two" in err.value
