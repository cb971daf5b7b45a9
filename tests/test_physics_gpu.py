"""Physics mode on the GPU through the C ABI against the FP64 oracle.

Tolerances (image NRMSE against FP64): FP32 panels 5e-5 (FP32 rounding of
t = ts + tg, ~1e-7 s, against the highest panel frequencies), BF16 panels
1e-3 (the gate the method is held to; 8 significant bits), FP16 panels
2.5e-4 (11 significant bits, each trace scaled by a power of two into FP16's
range).  Point-trace counts are exact.
"""
import numpy as np
import pytest

from tests.physics_case import engine, make_case, nrmse, oracle_run, records

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    c = make_case(nshots=2)
    c["o_img"], c["o_npt"], c["o_ints"] = oracle_run(c)
    assert np.abs(c["o_img"]).max() > 0
    return c


@pytest.mark.parametrize("dtype,tol", [(0, 5e-5), (1, 1e-3), (2, 2.5e-4)])
def test_image_nrmse(cuda, case, dtype, tol):
    eng, p, o = engine(case, panel_dtype=dtype)
    try:
        eng.submit(records(case))
        img = eng.get_image(False)
        _, npt = eng.counters()
    finally:
        eng.close()
    assert np.isfinite(img).all()
    assert npt == case["o_npt"]
    e = nrmse(img, case["o_img"])
    print(f"dtype {dtype}: NRMSE {e:.3e}")
    assert e <= tol


def test_kahan_and_batches(cuda, case):
    rec = records(case)
    eng, p, o = engine(case, kahan=1, max_batch=700)
    try:
        eng.submit(rec[:300])
        eng.submit(rec[300:])
        img = eng.get_image(False)
    finally:
        eng.close()
    assert nrmse(img, case["o_img"]) <= 5e-5


def test_block_and_little_endian(cuda):
    c = make_case(nshots=1, shots=[10], ixstart=30, ixend=100, half_x=60, half_y=40)
    ref, npt, _ = oracle_run(c)
    eng, p, o = engine(c)
    try:
        eng.submit(records(c, big_endian=False), big_endian=False)
        img = eng.get_image(False)
        _, n = eng.counters()
    finally:
        eng.close()
    assert n == npt
    assert nrmse(img, ref) <= 5e-5


def test_missing_tables_rejected(cuda, case):
    from q_psdm_b200 import engine as E
    eng, p, o = engine(case)
    try:
        sv = case["sv"]
        with pytest.raises(E.QpsdmError):
            eng.set_line(fxi=case["fxi"], cyi=case["cyi"],
                         dips=case["dips"].reshape(4, sv.nxi, sv.nzi))
        bad = case["tab"].as_engine_dict()
        bad["ttt"] = bad["ttt"][:100]
        with pytest.raises(E.QpsdmError):
            eng.set_line(fxi=case["fxi"], cyi=case["cyi"],
                         dips=case["dips"].reshape(4, sv.nxi, sv.nzi), tables=bad)
    finally:
        eng.close()


# ---- batched form ---------------------------------------------------------
@pytest.mark.parametrize("dtype,tol", [(0, 5e-5), (1, 1e-3), (2, 2.5e-4)])
@pytest.mark.parametrize("tile", [(32, 8), (64, 4), (16, 8), (32, 4)])
def test_batched_matches_fp64(cuda, case, dtype, tol, tile):
    eng, p, o = engine(case, panel_dtype=dtype, form=1, tile=tile)
    try:
        eng.submit(records(case))
        img = eng.get_image(False)
        _, npt = eng.counters()
    finally:
        eng.close()
    assert npt == case["o_npt"]
    assert nrmse(img, case["o_img"]) <= tol


def test_batched_many_shots_and_splits(cuda):
    # 11 shots exceed one source chunk (8 sources with the forced 32 x 4 tile);
    # irregular split
    c = make_case(shots=range(2, 13), rstep=8, half_x=50, half_y=40)
    ref, npt, _ = oracle_run(c)
    rec = records(c)
    eng, p, o = engine(c, form=1, max_batch=1000, kahan=1, tile=(32, 4))
    try:
        eng.submit(rec[:333])
        eng.submit(rec[333:])
        img = eng.get_image(False)
        _, n = eng.counters()
    finally:
        eng.close()
    assert n == npt
    assert nrmse(img, ref) <= 5e-5


def _varied_dips(case, seed=5, lo_hi=(0.05, 0.35)):
    """The case with dip limits that change from point to point (random
    tangents in [-0.35, -0.05] and [0.05, 0.35] by default, [-3, -2] and
    [2, 3] for steep limits), so that a tile's dip ranges matter."""
    c = dict(case)
    rng = np.random.default_rng(seed)
    n = case["dips"].shape[1]
    lo = -rng.uniform(*lo_hi, size=(2, n)).astype(np.float32)
    hi = rng.uniform(*lo_hi, size=(2, n)).astype(np.float32)
    c["dips"] = np.stack([lo[0], hi[0], lo[1], hi[1]])
    return c


def _image(c, **kw):
    eng, p, o = engine(c, **kw)
    try:
        eng.submit(records(c))
        img = eng.get_image(False)
        _, npt = eng.counters()
    finally:
        eng.close()
    return img, npt


@pytest.mark.parametrize("dips", ["reference", "varied", "steep"])
def test_batched_pointwise_equals_plain(cuda, case, dips):
    """The batched kernel drops, per image tile, the members whose dip test
    fails at every point of the tile (a conservative bound).  With FP32
    panels its image must then equal the plain form's point by point up to
    the order of the FP32 sums, for every tile shape, with the same
    point-trace count.  Varied dip limits also against the FP64 oracle;
    steep limits (tangents 2 to 3) exercise the bound's margin, which grows
    with the tangent."""
    c = {"reference": lambda: case, "varied": lambda: _varied_dips(case),
         "steep": lambda: _varied_dips(case, seed=6, lo_hi=(2.0, 3.0))}[dips]()
    plain, n0 = _image(c, panel_dtype=0, form=0)
    amp = np.abs(plain).max()
    assert amp > 0
    for tile in [(32, 8), (64, 4), (16, 8), (8, 16), (4, 32)]:
        img, n = _image(c, panel_dtype=0, form=1, tile=tile)
        assert n == n0, tile
        assert np.abs(img - plain).max() <= 2e-5 * amp, tile
    if dips != "reference":
        ref, npt, _ = oracle_run(c)
        assert n0 == npt
        assert nrmse(plain, ref) <= 5e-5


class _ShiftedQ:
    """Tables whose t* data sit behind a padding block, so that the t and t*
    descriptors differ (idx) while every value is the same."""

    def __init__(self, tab, pad=1000):
        self.tab, self.pad, self.dzii = tab, pad, tab.dzii

    def as_engine_dict(self):
        d = self.tab.as_engine_dict()
        dq = d["qqq_desc"].copy()
        dq[:, :8].view(np.int64)[:, 0] += self.pad
        d["qqq_desc"] = dq
        d["qqq"] = np.concatenate([np.full(self.pad, 7.0, np.float32), d["qqq"]])
        return d


def test_batched_unpaired_tables(cuda, case):
    """t and t* tables with different descriptors take the two-table lookup
    (identical descriptors are read as (t, t*) pairs): same image."""
    paired, n0 = _image(case, panel_dtype=0, form=1)
    c = dict(case)
    c["tab"] = _ShiftedQ(case["tab"])
    img, n = _image(c, panel_dtype=0, form=1)
    assert n == n0
    assert np.abs(img - paired).max() <= 1e-6 * np.abs(paired).max()


# ---- image bricks (several lines per submit) ------------------------------
@pytest.mark.parametrize("form,dtype,tol", [(0, 0, 5e-5), (1, 0, 5e-5), (1, 1, 1e-3)])
def test_brick_equals_single_lines(cuda, form, dtype, tol):
    base = make_case(nshots=2, rstep=2, half_y=40)
    lines = [58, 64, 70]
    refs, npt_ref = [], 0
    for L in lines:
        c = dict(base, line=L, cyi=base["sv"].line_y(L))
        img, npt, _ = oracle_run(c)
        refs.append(img)
        npt_ref += npt
    eng, p, o = engine(base, panel_dtype=dtype, form=form)
    try:
        sv = base["sv"]
        d = base["dips"].reshape(4, sv.nxi, sv.nzi)
        eng.set_lines([dict(fxi=base["fxi"], cyi=sv.line_y(L), dips=d,
                            tables=base["tab"].as_engine_dict()) for L in lines])
        eng.begin_offset(o)
        eng.submit(records(base))
        img = eng.get_image(False)
        _, npt = eng.counters()
    finally:
        eng.close()
    assert img.shape == (3, base["nxb"], sv.nzi)
    assert npt == npt_ref
    for k in range(3):
        assert nrmse(img[k], refs[k]) <= tol, k


@pytest.mark.parametrize("use_graph", [0, 1])
def test_brick_lines_on_two_streams_bit_identical(cuda, use_graph):
    """In the batched form the lines of a brick alternate between two
    streams, each with its own grouping buffers.  Every line's image and the
    counters must be bit-identical to that line imaged alone by an engine of
    its own (same kernels, same member order), eager or replayed from a
    captured graph; a line mask that skips lines keeps the alternation
    consistent."""
    base = make_case(nshots=2, rstep=2, half_y=40)
    sv = base["sv"]
    d = base["dips"].reshape(4, sv.nxi, sv.nzi)
    lines = [56, 60, 64, 68, 72]
    specs = [dict(fxi=base["fxi"], cyi=sv.line_y(L), dips=d,
                  tables=base["tab"].as_engine_dict()) for L in lines]
    rec = records(base)
    alone1, alone3, stats_alone = [], [], []
    for sp in specs:
        eng, p, o = engine(base, panel_dtype=2, form=1, variant=20)
        try:
            eng.set_lines([sp])
            eng.begin_offset(o)
            eng.submit(rec)
            alone1.append(eng.get_image(False))
            eng.submit(rec)
            eng.submit(rec)
            alone3.append(eng.get_image(False))
            stats_alone.append(eng.stats())
        finally:
            eng.close()
    eng, p, o = engine(base, panel_dtype=2, form=1, variant=20, use_graph=use_graph)
    try:
        eng.set_lines(specs)
        eng.begin_offset(o)
        for _ in range(3):   # eager, captured, replayed when use_graph
            eng.submit(rec)
        img = eng.get_image(False)
        st = eng.stats()
        # lines 1 and 3 only: the mask's two lines still alternate streams
        eng.begin_offset(o)
        eng.set_line_mask(0b01010)
        eng.submit(rec)
        masked = eng.get_image(False)
    finally:
        eng.close()
    for k in range(len(lines)):
        assert np.array_equal(img[k], alone3[k]), k
    for key in ("point_traces", "tile_decided", "imaged"):
        assert st[key] == sum(s[key] for s in stats_alone), key
    for k in range(len(lines)):
        want = alone1[k] if k in (1, 3) else np.zeros_like(alone1[k])
        assert np.array_equal(masked[k], want), k


def test_graph_replay_matches_eager(cuda):
    """use_graph: batches replayed from captured CUDA graphs give the same
    image as eager launches (same kernels, same order)."""
    c = make_case(nshots=2, rstep=2)
    rec = records(c)
    half = rec.shape[0] // 2
    imgs, counts = [], []
    for g in (0, 1):
        eng, p, o = engine(c, form=1, panel_dtype=1, use_graph=g, max_batch=half)
        try:
            for _ in range(2):          # a second pass replays the graphs
                eng.begin_offset(o)
                for k in range(3):      # eager, capture, replay of each buffer
                    eng.submit(rec[:half])
                    eng.submit(rec[half:2 * half])
            imgs.append(eng.get_image(False))
            counts.append(eng.counters())
        finally:
            eng.close()
    assert np.array_equal(imgs[0], imgs[1])
    # both counters are kept on the device: replays count like eager batches
    assert counts[0] == counts[1]
    ints = oracle_run(c)[2]
    acc = int((ints[:2 * half, 0] == 3).sum())
    assert counts[0][0] == 3 * acc


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("gain", [1e5, 1e-6])
def test_fp16_panels_any_amplitude(cuda, case, form, gain):
    """FP16 panels hold traces of any amplitude: the per-trace power-of-two
    scale keeps samples inside FP16's normal range (without it 1e5 overflows
    to inf and 1e-6 sinks into subnormals)."""
    c = dict(case, traces=(case["traces"] * np.float32(gain)).astype(np.float32))
    eng, p, o = engine(c, panel_dtype=2, form=form)
    try:
        eng.submit(records(c))
        img = eng.get_image(False) / gain
    finally:
        eng.close()
    assert np.isfinite(img).all()
    assert nrmse(img, case["o_img"]) <= 2.5e-4


@pytest.mark.parametrize("variant", list(range(1, 26)))
def test_every_batched_variant(cuda, case, variant):
    """Each launch variant the autotuner may pick (tile, blocks per SM, source
    chunk, the original or the compacted kernel) images the same as the FP64
    oracle."""
    eng, p, o = engine(case, panel_dtype=2, form=1, variant=variant)
    try:
        eng.submit(records(case))
        img = eng.get_image(False)
        _, npt = eng.counters()
        assert eng.tuning()["variant"] == variant - 1
    finally:
        eng.close()
    assert npt == case["o_npt"]
    assert nrmse(img, case["o_img"]) <= 2.5e-4


@pytest.mark.parametrize("orig,compact", [(11, 14), (13, 16), (2, 17), (9, 18)])
def test_compacted_kernel_counts_equal_original(cuda, case, orig, compact):
    """The compacted kernel (kept members listed in shared memory, uniform
    tiles counted in the keep pass) decides, counts and images exactly the
    pairs the original kernel does for the same tile shape, and its image
    agrees with the original's to FP32 rounding."""
    out = {}
    for v in (orig, compact):
        eng, p, o = engine(case, panel_dtype=2, form=1, variant=v)
        try:
            eng.submit(records(case))
            out[v] = (eng.get_image(False), eng.stats())
        finally:
            eng.close()
    (a, sa), (b, sb) = out[orig], out[compact]
    assert sa == sb
    assert nrmse(b, a) <= 1e-5


@pytest.mark.parametrize("fast,orig", [(14, 11), (20, 11), (23, 11), (22, 13), (16, 13), (17, 2),
                                       (24, 11), (25, 11)])
def test_fast_form_defers_straddling_tiles(cuda, fast, orig):
    """An image block starting at cdp 30 puts table-cell edges (every 16 cdps)
    inside tiles: the fast form leaves those tiles to the original kernel
    (a device list of tiles), and the image and every counter equal the
    original kernel's alone and the FP64 oracle's point-traces."""
    c = make_case(nshots=2, ixstart=30, ixend=126)
    ref, npt, _ = oracle_run(c)
    out = {}
    for v in (orig, fast):
        eng, p, o = engine(c, panel_dtype=2, form=1, variant=v)
        try:
            eng.submit(records(c))
            out[v] = (eng.get_image(False), eng.stats())
        finally:
            eng.close()
    (a, sa), (b, sb) = out[orig], out[fast]
    assert sb["point_traces"] == npt
    assert sa == sb
    assert nrmse(b, a) <= 1e-5
    assert nrmse(b, ref) <= 2.5e-4


@pytest.mark.parametrize("scalar,packed", [(20, 24), (20, 25)])
def test_packed_walk_equals_scalar_walk(cuda, scalar, packed):
    """The walk on packed FP32 pairs (two members per f32x2 instruction)
    images exactly the pairs the scalar walk images -- every deciding value
    is the same IEEE operation -- with equal counters and the image equal to
    FP32 rounding, FP16 and FP32 panels, also with tiles left to the
    original kernel (an image block starting at cdp 30) and Kahan sums."""
    for c, kw in ((make_case(nshots=2), dict(panel_dtype=2)),
                  (make_case(nshots=2), dict(panel_dtype=0, kahan=1)),
                  (make_case(nshots=2, ixstart=30, ixend=126), dict(panel_dtype=2))):
        out = {}
        for v in (scalar, packed):
            eng, p, o = engine(c, form=1, variant=v, **kw)
            try:
                eng.submit(records(c))
                out[v] = (eng.get_image(False), eng.stats())
            finally:
                eng.close()
        (a, sa), (b, sb) = out[scalar], out[packed]
        assert sa == sb
        assert np.abs(b - a).max() <= 1e-6 * np.abs(a).max()
