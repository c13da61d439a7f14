"""Helpers shared by the tests (host-side conversions and comparisons)."""
import numpy as np


def tiled_to_linear(a, nx, ny, nz):
    """Tile-blocked slot array (slot = tile*512 + (i&7) + 8(j&7) + 64(k&7)) ->
    x-fastest linear array of nx*ny*nz."""
    tx, ty = nx // 8, ny // 8
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    tile = (i >> 3) + tx * ((j >> 3) + ty * (k >> 3))
    slot = tile * 512 + (i & 7) + 8 * (j & 7) + 64 * (k & 7)
    return np.asarray(a)[slot.ravel()]


def rel_err(a, b, floor=0.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = max(np.max(np.abs(b)), floor)
    if den == 0.0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / den)


def u32(t):
    """torch int32 tensor holding u32 bits -> numpy uint32."""
    return t.cpu().numpy().view(np.uint32)
