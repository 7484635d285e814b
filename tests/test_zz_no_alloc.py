"""The allocation-free even-odd operator (hw_wilson_evenodd_apply_noalloc).

It exists for callers that cannot call cudaMalloc (a framework's pool owns the
device memory, or allocation is not allowed where they run), so it takes its
temporary field from a fixed array inside the library.  This test lays out
links and spinors in the library's even-odd device layout with numpy, puts them
on the GPU with torch (the caller's allocator), calls the entry point twice in
a row through the C ABI, and checks each output against the normal
hw_wilson_evenodd_apply / dagger on the same input and against the CPU oracle,
to the operator tolerance 1e-13 per site, for both link formats and both time
boundary conditions.  This file is collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SITE_TOL = 1e-13


def eo_index(dims):
    """checkerboard order: for parity p, lex indices sorted by lex // 2."""
    Lx, Ly, Lz, Lt = dims
    lex = np.arange(Lx * Ly * Lz * Lt)
    x = lex % Lx
    y = (lex // Lx) % Ly
    z = (lex // (Lx * Ly)) % Lz
    t = lex // (Lx * Ly * Lz)
    par = (x + y + z + t) % 2
    return [lex[par == p] for p in (0, 1)]  # ascending lex -> checkerboard index lex // 2


def spinor_planes(psi, sites, stride):
    """(V,4,3,2) -> (12, stride) complex planes (double2) of the given parity."""
    c = psi.reshape(-1, 12, 2)[sites]
    out = np.zeros((12, stride, 2))
    out[:, :len(sites)] = c.transpose(1, 0, 2)
    return out


def link_planes(U, idx, stride, link_format=18):
    """(4,V,3,3,2) -> ((par*4+dir)*planes + k, stride) double2 planes: 9 planes (18 reals)
    or the first two rows in 6 planes (12 reals; the third row is rebuilt on the GPU)."""
    planes = 9 if link_format == 18 else 6
    out = np.zeros((2, 4, planes, stride, 2))
    Uc = U.reshape(4, -1, 9, 2)[:, :, :planes]
    for p in (0, 1):
        for d in range(4):
            out[p, d, :, :len(idx[p])] = Uc[d, idx[p]].transpose(1, 0, 2)
    return out.reshape(-1, stride, 2)


def rel_site_err(a, b):
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    return np.where(den > 0, num / np.maximum(den, 1e-300), num).max()


@pytest.mark.parametrize("link_format", [18, 12])
@pytest.mark.parametrize("antiperiodic", [True, False])
def test_noalloc_matches_evenodd_apply(hw, ctx, oracle, link_format, antiperiodic):
    import torch
    dims = (8, 4, 4, 8)
    kappa = 0.124
    V = int(np.prod(dims))
    stride = V // 2 + 64  # any stride >= sites per parity
    idx = eo_index(dims)
    U = oracle.gen_links(dims, 0.3, 77)
    lat = hw.Lattice(ctx, dims, antiperiodic)
    G = hw.GaugeField(lat, U, link_format)
    D = hw.Dirac_Wilson_evenodd(kappa, G)
    dev = torch.device("cuda:0")
    links_d = torch.from_numpy(np.ascontiguousarray(link_planes(U, idx, stride, link_format))).to(dev)
    out_d = torch.zeros((12, stride, 2), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (seed, sign) in enumerate([(78, 1), (79, -1)]):
        psi = oracle.gen_spinor(dims, seed, oracle.EVEN)
        in_d = torch.from_numpy(np.ascontiguousarray(spinor_planes(psi, idx[0], stride))).to(dev)
        torch.cuda.synchronize()
        hw.wilson_evenodd_apply_noalloc(dims, kappa, sign, links_d.data_ptr(), in_d.data_ptr(), out_d.data_ptr(),
                                        stride, link_format=link_format, antiperiodic=antiperiodic, stream=stream)
        torch.cuda.synchronize()
        got = out_d.cpu().numpy()[:, :len(idx[0])].transpose(1, 0, 2).reshape(-1, 24)
        fin, fout = hw.Field(lat, psi), hw.Field(lat)
        (D.apply if sign > 0 else D.dagger)(fin, fout)
        ref = fout.download().reshape(-1, 24)[idx[0]]
        assert rel_site_err(got, ref) <= SITE_TOL, f"call {call}: against hw_wilson_evenodd_apply"
        ora = oracle.eo_apply(dims, U, kappa, psi, sign, antiperiodic).reshape(-1, 24)[idx[0]]
        assert rel_site_err(got, ora) <= SITE_TOL, f"call {call}: against the oracle"
        for f in (fin, fout):
            f.close()
    for h in (G, lat):
        h.close()


def test_noalloc_rejects_large_lattice(hw, ctx):
    with pytest.raises(hw.HilaError) as e:
        hw.wilson_evenodd_apply_noalloc((16, 16, 16, 18), 0.12, 1, 0x1000, 0x1000, 0x1000, 1 << 20)
    assert e.value.code == hw.HW_ERR_INVALID
    assert "at most 32768" in str(e.value)
    # extents whose product would overflow are rejected as soon as the running product is too large
    with pytest.raises(hw.HilaError) as e:
        hw.wilson_evenodd_apply_noalloc((1 << 30, 1 << 30, 1 << 30, 1 << 30), 0.12, 1, 0x1000, 0x1000, 0x1000,
                                        1 << 20)
    assert e.value.code == hw.HW_ERR_INVALID and "at most 32768" in str(e.value)
