"""Host logic of configuration 4's evaluation (no GPU): the evaluated source
positions lie between solved sources, their four corners are solved sources,
and every evaluated node is a node of all five grids involved -- the
position's own and the corners' (each n x n x nz, spacing h, centred on its
source) -- so the solver's values can be read there without interpolation."""
import numpy as np
import pytest

from q_psdm_b200 import surrogate as S


@pytest.mark.parametrize("n_side,spacing,stride,n,nz,h", [
    (64, 80.0, 8, 64, 51, 40.0),     # the GPU test's scale
    (64, 80.0, 2, 128, 101, 40.0),   # the bench's default scale
    (64, 80.0, 1, 256, 201, 20.0),   # the full configuration
])
def test_evaluation_nodes_lie_on_all_five_grids(n_side, spacing, stride, n, nz, h):
    hx, hy, ix, iy, step, corners, nodes = S.config4_eval_points(
        n_side=n_side, spacing=spacing, stride=stride, n=n, nz=nz, h=h, held=16,
        held_nodes=2048, seed=3)
    held = hx.size
    solved = S.source_grid(n_side, spacing)[
        np.repeat(np.arange(n_side) % stride == 0, n_side)
        & np.tile(np.arange(n_side) % stride == 0, n_side)]
    solved_set = {(float(x), float(y)) for x, y in solved}
    for c in corners:
        assert (float(c[0]), float(c[1])) in solved_set
    for k in range(held):
        assert ix[k] * step <= hx[k] <= (ix[k] + 1) * step
        assert iy[k] * step <= hy[k] <= (iy[k] + 1) * step
        srcs = [(hx[k], hy[k])] + [tuple(corners[c * held + k]) for c in range(4)]
        p = nodes[k]
        for sx, sy in srcs:
            o = S._local_origin(np.array([[sx, sy]]), n, h)[0]
            li = (p[:, 0] - o[0]) / h
            lj = (p[:, 1] - o[1]) / h
            lk = p[:, 2] / h
            for v, top in ((li, n), (lj, n), (lk, nz)):
                assert np.allclose(v, np.rint(v), atol=1e-3)   # on the lattice
                assert v.min() >= 0 and v.max() <= top - 1
