"""GB energy through the entry point that allocates no device memory.

Callers that cannot allocate (their device memory belongs to a host
framework's allocator, or they run in loops that must not enter the driver's
allocator) use rstg_gb_energy_noalloc_async with their own device buffers.
This test calls it through the C ABI and checks it against the allocating
entry point, rstg_gb_energy_compute, with the tolerances of the other GB
parity tests (relative 1e-10 on the energy, 1e-12 on Born radii), over calls
in a row of different sizes and models -- the scratch array is shared by all
calls -- including an odd atom count (the last warp's pair rows are split
unevenly) and calls enqueued on a caller-created stream, and checks that an
oversized request is refused.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(tmp_path, name, n_rec, n_lig, seed):
    import rust_simulation_tools as rst
    from rust_simulation_tools import synthetic as S

    s = S.make_system(n_rec, n_lig, seed=seed)
    fr = S.make_frames(s, 1, seed=seed + 1)
    p = str(tmp_path / f"{name}.prmtop")
    S.write_prmtop(s, p)
    x = (fr[0].astype(np.float64) * 0.1) * 10.0
    return rst.read_prmtop(p), x


def test_noalloc_gb_matches_allocating_entry_point(tmp_path):
    import torch

    import rust_simulation_tools as rst
    from rust_simulation_tools import _native as N

    if rst.device_count() < 1 or not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    side = torch.cuda.Stream()
    cases = [
        ("a", 300, 24, 41, rst.GbParams(model=rst.GbModel.ObcII, solvent_dielectric=78.5), None),
        ("b", 90, 10, 43, rst.GbParams(model=rst.GbModel.Hct, salt_concentration=0.0), None),
        ("a", 300, 24, 41, rst.GbParams(model=rst.GbModel.ObcI), side),
        ("c", 97, 10, 47, rst.GbParams(model=rst.GbModel.ObcII), side),  # 107 atoms
        ("c", 97, 10, 47, rst.GbParams(model=rst.GbModel.ObcI, salt_concentration=0.0), None),
    ]
    for name, nr, nl, seed, params, stream in cases:
        top, x = _case(tmp_path, name, nr, nl, seed)
        ref = rst.compute_gb_energy(top, x / 10.0, params)
        atoms = top._atoms()
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
        d_x, d_q, d_r, d_s = dev(x * 1.0), dev(atoms["charges_amber"]), dev(atoms["radii"]), dev(atoms["screen"])
        n = len(x)
        d_total = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        d_born = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        ptr = lambda t: N.vp(t.data_ptr())
        torch.cuda.synchronize()  # inputs are ready before a side stream reads them
        for keep_radii in (True, False):
            rc = N.lib.rstg_gb_energy_noalloc_async(ptr(d_x), ptr(d_q), ptr(d_r), ptr(d_s), n, C.byref(params._c),
                                                   ptr(d_total), ptr(d_born) if keep_radii else None,
                                                   N.vp(stream.cuda_stream) if stream is not None else None)
            N.check(rc)
            if stream is not None:
                stream.synchronize()
            else:
                torch.cuda.synchronize()
            total = float(d_total.cpu()[0])
            assert abs(total - ref.total) <= 1e-10 * max(1.0, abs(ref.total)), (name, keep_radii, total, ref.total)
            if keep_radii:
                np.testing.assert_allclose(d_born.cpu().numpy(), ref.born_radii(), rtol=1e-12)
    rc = N.lib.rstg_gb_energy_noalloc_async(ptr(d_x), ptr(d_q), ptr(d_r), ptr(d_s), 131073, None, ptr(d_total),
                                           None, None)
    assert rc == N.ERR_INVALID
    assert "131072" in N.lib.rstg_last_error().decode()
