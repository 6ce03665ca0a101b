"""Column form of the 3D coefficient volumes (engine.coef_columns): the fused
step reads repeated (x, z) columns from a small table, so the table plus the
volumes where ctype == 255 must give back every coefficient bit for bit."""
import numpy as np
import torch

from lens_sensor_b200.engine import coef_columns


def _vols(ncoef, nx=40, ny=30, nz=50, P=64, seed=0):
    rng = np.random.default_rng(seed)
    colA = rng.random((6, ny)).astype(np.float32)
    colB = rng.random((6, ny)).astype(np.float32)
    vols = [torch.zeros((nx, ny, P)) for _ in range(ncoef)]
    for c, v in enumerate(vols):
        v[:, :, :nz] = torch.from_numpy(colA[c])[None, :, None]
        v[:10, :, :nz] = torch.from_numpy(colB[c])[None, :, None]
        v[20:25, 5:9, 10:14] = torch.from_numpy(rng.random((5, 4, 4)).astype(np.float32))   # a bead patch
        v[33, 7, 3] = float(np.nextafter(np.float32(v[33, 7, 3]), np.float32(2.0)))          # one ulp off
    return vols, nx, ny, nz


def _rebuild(vols, cols, nz):
    ct, tab, ex, nt = cols
    for c, v in enumerate(vols):
        rec = torch.where(ct[:, None, :] == 255, v, tab[ct.clamp(max=nt - 1).long(), c].permute(0, 2, 1))
        assert torch.equal(rec[:, :, :nz].view(torch.int32), v[:, :, :nz].view(torch.int32)), c


def test_columns_rebuild_every_coefficient_exactly():
    for ncoef in (3, 6):
        vols, nx, ny, nz = _vols(ncoef)
        cols = coef_columns(vols, nx, ny, nz, min_count=8)
        assert cols is not None and cols[3] == 2
        ct, tab, ex, nt = cols
        assert ct[33, 3] == 255                          # the column one ulp off keeps its volume values
        assert int((ct[:, :nz] == 255).sum()) == 5 * 4 + 1
        # the explicit flag marks exactly the 32-column groups holding a type-255 column
        want = (ct == 255).view(nx, -1, 32).any(dim=2)
        assert torch.equal(ex.bool(), want)
        _rebuild(vols, cols, nz)


def test_no_repeated_columns_gives_no_table():
    rng = np.random.default_rng(1)
    vols = [torch.from_numpy(rng.random((8, 6, 32)).astype(np.float32)) for _ in range(3)]
    assert coef_columns(vols, 8, 6, 20) is None
