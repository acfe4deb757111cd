"""Compact trees on the host (no GPU): the oracle's restatement of
SceneBuilder's compaction (vulkan/src/engine/scene_builder.cpp: BuildNode
:91-156, LayoutNode :199-238) and the library's blob format (frep.compact:
pack / expand, and frep_compact_check, which needs no device)."""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from frep import compact, scenes
from frep._lib import ERR_INVALID_ARG, FrepError


def _oracle(sc, rounding=1):
    tape = frep.Tape(sc.shape)
    return oracle.OracleTree(tape.wide(), tape.n_slots, sc.grid_dims, sc.low_vertex, sc.world_size,
                             rounding=rounding, threads=8)


@pytest.fixture(scope="module")
def spheres():
    return _oracle(scenes.spheres_union(16, seed=1, width=96, height=96))


@pytest.fixture(scope="module")
def three_level():
    return _oracle(scenes.random_csg(24, seed=5, grid_dims=[8, 4, 4], width=96, height=64))


def _records(t, l):
    return t.nodes[t.node_offset[l]: t.node_offset[l] + t.node_count[l] * t.node_size[l]].reshape(
        t.node_count[l], t.node_size[l])


def _solid(t) -> np.ndarray:
    """Finest-grid occupancy: every leaf cell of every node, expanded."""
    fine = int(np.prod(t.dims))
    occ = np.zeros((fine, fine, fine), bool)
    for l, dim in enumerate(t.dims):
        span = int(np.prod(t.dims[l + 1:]))
        for rec in _records(t, l):
            cells = compact._cells(rec[4:4 + dim ** 3 // 32])
            x0, y0, z0 = (int(v) * dim for v in rec[1:4])
            for c in cells:
                x, y, z = x0 + c // (dim * dim), y0 + (c // dim) % dim, z0 + c % dim
                occ[x * span:(x + 1) * span, y * span:(y + 1) * span, z * span:(z + 1) * span] = True
    return occ


def _children_in_preorder(t) -> bool:
    """Children of consecutive nodes are consecutive, each in cell order."""
    for l in range(t.levels - 1):
        c3 = t.dims[l] ** 3
        ids = [rec[4 + c3 // 16 + compact._cells(rec[4 + c3 // 32:4 + c3 // 16])] for rec in _records(t, l)]
        ids = np.concatenate(ids) if ids else np.zeros(0)
        if not np.array_equal(ids, np.arange(t.node_count[l + 1])):
            return False
    return True


@pytest.mark.parametrize("which", ["spheres", "three_level"])
def test_layout_keeps_every_node_in_preorder(which, request):
    src = request.getfixturevalue(which)
    c = src.compact(prune=False)
    assert c.node_count == src.node_count
    a, pa = oracle.canonical_of_oracle(src)
    b, pb = oracle.canonical_of_oracle(c)
    assert pa == [] and pb == [] and a == b
    assert _children_in_preorder(c)


@pytest.mark.parametrize("which", ["spheres", "three_level"])
def test_prune_applies_buildnode_rules(which, request):
    src = request.getfixturevalue(which)
    p = src.compact(prune=True)
    assert _children_in_preorder(p)
    assert oracle.canonical_of_oracle(p)[1] == []
    np.testing.assert_array_equal(_solid(p), _solid(src))
    # no node below the root is empty or has only leaf cells
    for l in range(1, p.levels):
        w = p.dims[l] ** 3 // 32
        last = l == p.levels - 1
        for rec in _records(p, l):
            leaf = rec[4:4 + w]
            inter = np.zeros(w, np.uint32) if last else rec[4 + w:4 + 2 * w]
            assert (leaf | inter).any()
            assert not (leaf == 0xFFFFFFFF).all()
    assert sum(p.node_count) <= sum(src.node_count)


def test_pruning_removes_nodes_somewhere(three_level):
    p = three_level.compact(prune=True)
    assert sum(p.node_count) < sum(three_level.node_count)


def test_layout_renders_like_the_source(spheres):
    sc = scenes.spheres_union(16, seed=1, width=96, height=96)
    c = spheres.compact(prune=False)
    cam = oracle.camera_vector(sc.camera, 96, 96)
    lights = frep.Lights(shadow_mask=1)
    ra, ha = spheres.render(cam, lights)
    rb, hb = c.render(cam, lights)
    np.testing.assert_array_equal(ra, rb)
    ka = oracle.hit_cells(ha, spheres.dims, spheres.node_offset, spheres.node_size, spheres.nodes)
    kb = oracle.hit_cells(hb, c.dims, c.node_offset, c.node_size, c.nodes)
    np.testing.assert_array_equal(ka, kb)
    np.testing.assert_array_equal(ha[..., :4], hb[..., :4])  # depth and normal bits


@pytest.mark.parametrize("which", ["spheres", "three_level"])
def test_pack_expand_round_trip(which, request):
    src = request.getfixturevalue(which)
    blob = compact.pack(src.levels, src.dims, src.node_count, src.node_offset, src.node_size, src.nodes,
                        src.tapes, src.low_vertex, src.world_size, src.n_slots)
    compact.check(blob)
    e = compact.expand(blob)
    want = src.compact(prune=False)
    assert e.node_count == want.node_count
    assert e.node_size == want.node_size
    np.testing.assert_array_equal(e.nodes, want.nodes)
    np.testing.assert_array_equal(e.tapes, want.tapes)
    again = compact.pack(e.levels, e.dims, e.node_count, e.node_offset, e.node_size, e.nodes, e.tapes,
                         e.low_vertex, e.world_size, e.n_slots)
    np.testing.assert_array_equal(again, blob)


def test_pruned_tree_packs_to_a_valid_blob(three_level):
    p = three_level.compact(prune=True)
    blob = compact.pack(p.levels, p.dims, p.node_count, p.node_offset, p.node_size, p.nodes, p.tapes,
                        p.low_vertex, p.world_size, p.n_slots)
    compact.check(blob)
    np.testing.assert_array_equal(compact.expand(blob).nodes, p.nodes)


def _expect_invalid(blob, what):
    with pytest.raises(FrepError) as ei:
        compact.check(blob)
    assert ei.value.status == ERR_INVALID_ARG, what


def test_check_rejects_damaged_blobs(three_level):
    t = three_level
    good = compact.pack(t.levels, t.dims, t.node_count, t.node_offset, t.node_size, t.nodes, t.tapes,
                        t.low_vertex, t.world_size, t.n_slots)
    compact.check(good)
    b = compact.parse(good)
    w0 = t.dims[0] ** 3 // 32
    nat = 120  # node section offset

    def patched(word_index, value, dtype=np.uint32, at=nat):
        out = good.copy()
        out[at + word_index * np.dtype(dtype).itemsize: at + (word_index + 1) * np.dtype(dtype).itemsize] = \
            np.array([value], dtype).view(np.uint8)
        return out

    bad = good.copy()
    bad[0] = ord("X")
    _expect_invalid(bad, "magic")
    _expect_invalid(good[:-8], "truncated")
    _expect_invalid(np.concatenate([good, np.zeros(8, np.uint8)]), "trailing bytes")
    _expect_invalid(good[:100], "shorter than the header")
    # header fields (byte offsets of frep_compact_header)
    _expect_invalid(patched(0, 2, at=8), "version")
    _expect_invalid(patched(0, 9, at=12), "levels")
    _expect_invalid(patched(0, 6, at=16), "dims[0] not a multiple of 4")
    _expect_invalid(patched(0, 2000, at=68), "n_slots")
    _expect_invalid(patched(0, 2, at=72), "two roots")
    # root record: [tape, leaf[W], interior[W], prefix[W], base]
    inter = b.nodes[1 + w0:1 + 2 * w0]
    wi = int(np.nonzero(inter)[0][0])
    _expect_invalid(patched(1 + 2 * w0 + wi + 1, int(b.nodes[1 + 2 * w0 + wi + 1]) + 1), "prefix")
    _expect_invalid(patched(1 + 3 * w0, 1), "base")
    _expect_invalid(patched(1 + wi, int(b.nodes[1 + wi]) | int(inter[wi])), "leaf and interior")
    _expect_invalid(patched(0, len(b.tapes) + 16), "tape index")
    # a tape instruction with an out-of-range slot
    tat = 120 + (4 * len(b.nodes) + 7) // 8 * 8
    n = int(b.tapes[0] & 0xFFFFFFFF)
    assert n > 0
    w = int(b.tapes[1]) & ~(0xFFFF << 16) | ((t.n_slots + 3) << 16)
    _expect_invalid(patched(1, w, np.uint64, at=tat), "slot")
    # a record that runs past the pool
    _expect_invalid(patched(0, (1 << 31), np.uint64, at=tat), "record length")


@pytest.mark.parametrize("rounding", [0, 1])
@pytest.mark.parametrize("which", ["spheres", "three_level"])
def test_tree_occupancy_equals_scenebuilder_point_sampling(which, rounding):
    """SceneBuilder::BuildNode (scene_builder.cpp:91-156) decides every
    finest voxel by the point value at its low corner,
    WorldPosition = lowVertex + pos * worldSize / fineGridDim
    (voxel_storage.h:58-61), through csg::Tape::Eval at T = 0. The interval
    tree (leaf cells at any level, expanded) must give the same solid set.
    The reference's own Tape::Eval is used where the reference bridge is built;
    elsewhere frep_tape_eval, which is pinned bit-exact to it."""
    sc = (scenes.spheres_union(16, seed=1, width=96, height=96) if which == "spheres"
          else scenes.random_csg(24, seed=5, grid_dims=[8, 4, 4], width=96, height=64))
    t = _oracle(sc, rounding)
    occ = _solid(t)
    fine = occ.shape[0]
    ii = np.indices(occ.shape).reshape(3, -1).T.astype(np.float32)
    low = np.asarray(sc.low_vertex, np.float32)
    pos = (low + (ii * np.float32(sc.world_size)) / np.float32(fine)).astype(np.float32)
    xyzt = np.concatenate([pos, np.zeros((len(pos), 1), np.float32)], 1)
    if oracle.ref_available():
        values = oracle.RefTape(*sc.shape.flatten()).eval(xyzt)
    else:
        values = frep.Tape(sc.shape).eval_points(xyzt)
    np.testing.assert_array_equal(occ, (values < 0).reshape(occ.shape))
    assert occ.sum() > 1000


def _safe_to_render(blob) -> bool:
    """The conditions the renderer relies on, restated independently: every
    interior cell's child index and every node's tape record (and each
    instruction's slots) lie inside their pools."""
    b = compact.parse(blob)
    if b.node_count[0] != 1 or not (4 <= b.n_slots <= 1024):
        return False
    sizes, offs = b.node_size, b.node_offset
    if offs[-1] + b.node_count[-1] * sizes[-1] != len(b.nodes):
        return False
    tw = len(b.tapes)
    for l in range(b.levels):
        w = b.dims[l] ** 3 // 32
        last = l == b.levels - 1
        recs = b.nodes[offs[l]: offs[l] + b.node_count[l] * sizes[l]].reshape(b.node_count[l], sizes[l])
        for rec in recs:
            t = int(rec[0])
            if t >= tw:
                return False
            n = int(b.tapes[t] & 0xFFFFFFFF)
            if t + 1 + n > tw:
                return False
            ins = b.tapes[t + 1: t + 1 + n]
            op = ins & 0xFF
            slots = np.stack([(ins >> 16) & 0xFFFF, (ins >> 32) & 0xFFFF, ins >> 48])
            if (op > 12).any() or (slots[0] >= b.n_slots).any() or \
                    ((op != 0) & ((slots[1] >= b.n_slots) | (slots[2] >= b.n_slots))).any():
                return False
            if last:
                continue
            inter = rec[1 + w:1 + 2 * w]
            cells = compact._cells(inter)
            if len(cells):
                words, bits = cells // 32, cells % 32
                below = np.bitwise_count(inter[words] & ((np.uint64(1) << bits.astype(np.uint64)) - 1).astype(np.uint32))
                child = rec[1 + 3 * w].astype(np.int64) + rec[1 + 2 * w + words].astype(np.int64) + below
                if (child >= b.node_count[l + 1]).any():
                    return False
    return True


def test_check_never_accepts_an_unsafe_blob(three_level):
    """Random word overwrites in the node and tape sections of a valid blob:
    whatever frep_compact_check accepts must be safe to render."""
    t = three_level
    good = compact.pack(t.levels, t.dims, t.node_count, t.node_offset, t.node_size, t.nodes, t.tapes,
                        t.low_vertex, t.world_size, t.n_slots)
    assert _safe_to_render(good)
    rng = np.random.default_rng(7)
    words = good[120:].view(np.uint32)
    accepted = 0
    for _ in range(400):
        bad = good.copy()
        bw = bad[120:].view(np.uint32)
        i = int(rng.integers(len(words)))
        bw[i] = rng.choice([0, 1, 0xFFFFFFFF, int(words[i]) ^ (1 << int(rng.integers(32))),
                            int(rng.integers(1 << 32))])
        try:
            compact.check(bad)
        except FrepError as e:
            assert e.status == ERR_INVALID_ARG
            continue
        accepted += 1
        assert _safe_to_render(bad), i
    assert accepted > 0  # some overwrites are harmless (leaf masks, instruction constants)


def test_save_and_load(three_level, tmp_path):
    t = three_level
    blob = compact.pack(t.levels, t.dims, t.node_count, t.node_offset, t.node_size, t.nodes, t.tapes,
                        t.low_vertex, t.world_size, t.n_slots)
    compact.save(blob, tmp_path / "tree.frepct")
    np.testing.assert_array_equal(compact.load(tmp_path / "tree.frepct"), blob)
    (tmp_path / "bad.frepct").write_bytes(bytes(blob[:-8]))
    with pytest.raises(FrepError):
        compact.load(tmp_path / "bad.frepct")


def test_save_and_check_reinterpret_word_arrays(three_level, tmp_path):
    """A blob held as u32 or u64 words is the same bytes: save() and check()
    reinterpret it instead of converting each word to a byte."""
    t = three_level
    blob = compact.pack(t.levels, t.dims, t.node_count, t.node_offset, t.node_size, t.nodes, t.tapes,
                        t.low_vertex, t.world_size, t.n_slots)
    assert blob.nbytes % 8 == 0
    for words in (blob.view(np.uint32), blob.view(np.uint64)):
        compact.check(words)
        compact.save(words, tmp_path / "w.frepct")
        np.testing.assert_array_equal(compact.load(tmp_path / "w.frepct"), blob)
