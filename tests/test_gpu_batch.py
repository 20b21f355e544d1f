"""Batched build + trace of many uneven triangle scenes (srt_batch_*) against
the per-scene plain path and the CPU oracle: hits bit-exact, prim ids local
to each scene, identical through autotuning, graph capture and replay."""
import numpy as np
import pytest
import torch

import surface_b200 as sb
from oracle import oracle as O
from surface_b200 import scenes as S
from surface_b200.batch import TriangleBatch

from conftest import bits

pytestmark = pytest.mark.gpu


def to_dev(B):
    return (torch.as_tensor(B["vertices"]).cuda(),
            torch.as_tensor(B["faces"].view(np.int32)).cuda(),
            torch.as_tensor(B["rays"].view(np.float32).reshape(-1, 8)).cuda())


def hits_np(h):
    return h.cpu().numpy().reshape(-1).view(sb.HIT_DTYPE)


def per_scene(B, v, f, r):
    """The plain loop: one TriangleAccel build + trace per scene."""
    fo, ro = B["face_offsets"], B["ray_offsets"]
    out = []
    for s in range(fo.size - 1):
        acc = sb.TriangleAccel()
        acc.Build32(sb.Mesh(v, f[int(fo[s]):int(fo[s + 1])]))
        out.append(hits_np(acc.Traverse(r[int(ro[s]):int(ro[s + 1])])))
        acc.close()
    return np.concatenate(out)


def assert_same(a, b):
    for k in ("t", "u", "v", "prim"):
        bad = np.nonzero(bits(a[k]) != bits(b[k]))[0]
        assert bad.size == 0, f"{k}: {bad.size} mismatches, first at {bad[:5]}"


def small_batch(seed=7, n=12):
    return S.batched_scenes(n, seed=seed, lo=1e3, hi=4e4, sizes=(16, 32, 48), min_faces=2)


def test_batch_matches_per_scene_and_oracle():
    B = small_batch()
    v, f, r = to_dev(B)
    tb = TriangleBatch()
    h = hits_np(tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"]))
    torch.cuda.synchronize()
    assert_same(h, per_scene(B, v, f, r))
    assert (h["prim"] != sb.MISS).any()
    fo, ro = B["face_offsets"], B["ray_offsets"]
    for s in (0, 5, 11):
        faces = B["faces"][int(fo[s]):int(fo[s + 1])]
        ref = O.OracleAccel(O.TRI, B["vertices"], faces).trace(
            B["rays"][int(ro[s]):int(ro[s + 1])])
        assert_same(h[int(ro[s]):int(ro[s + 1])], ref)
        hit = h["prim"][int(ro[s]):int(ro[s + 1])]
        assert hit[hit != sb.MISS].max() < faces.shape[0]  # scene-local ids


def test_graph_capture_and_replay_are_identical():
    B = small_batch(seed=9, n=20)
    v, f, r = to_dev(B)
    tb = TriangleBatch()
    first = hits_np(tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"]))
    blk, R, captured, kpc = tb.config()
    assert blk in (64, 128, 256) and R in (1, 2, 4) and not captured
    for call in range(4):
        h = torch.full((r.shape[0], 4), float("nan"), device="cuda")
        # same output tensor each time after the first: capture needs equal args
        h = tb._keep[3] if call else h
        h.fill_(float("nan"))
        out = hits_np(tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"], hits=h))
        assert_same(out, first)
    assert tb.config()[2], "third identical call should replay a captured graph"
    assert tb.config()[3] == kpc


@pytest.mark.parametrize("depth", [24, 32, 48])
@pytest.mark.parametrize("sort_bits", [0, 12, 22])
def test_every_tuning_point_gives_the_same_hits(depth, sort_bits):
    """The autotuner's axes -- stack depth and ray order -- pinned one point at
    a time: the same hits as the per-scene path, through capture and replay."""
    B = small_batch(seed=5, n=10)
    v, f, r = to_dev(B)
    want = per_scene(B, v, f, r)
    tb = TriangleBatch()
    tb.set_tuning(block=64 if sort_bits else 256, rays_per_grab=2, stack_depth=depth,
                  sort_bits=sort_bits)
    hits = torch.empty((r.shape[0], 4), device="cuda")
    for _ in range(3):
        hits.fill_(float("nan"))
        assert_same(hits_np(tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"],
                                           hits=hits)), want)
    assert tb.config()[2]
    assert tb.tuning() == {"block": 64 if sort_bits else 256, "rays_per_grab": 2,
                           "stack_depth": depth, "sort_bits": sort_bits}


def test_autotuned_point_is_reported():
    B = small_batch(seed=8, n=8)
    v, f, r = to_dev(B)
    tb = TriangleBatch()
    tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"])
    t = tb.tuning()
    assert t["block"] in (64, 128, 256) and t["rays_per_grab"] in (1, 2, 4)
    assert t["stack_depth"] in (24, 32, 48) and t["sort_bits"] in (0, 12, 22)
    with pytest.raises(sb.SurfaceError):
        tb.set_tuning(stack_depth=40)


def test_replay_sees_new_input_values():
    """A replay reads the buffers again: moved vertices give new hits."""
    B = small_batch(seed=3, n=6)
    v, f, r = to_dev(B)
    tb = TriangleBatch()
    hits = torch.empty((r.shape[0], 4), device="cuda")
    for _ in range(3):
        tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"], hits=hits)
    assert tb.config()[2]
    v.mul_(0.5)  # shrink every scene in place
    out = hits_np(tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"], hits=hits))
    assert_same(out, per_scene(B, v, f, r))


def test_changed_arguments_recapture():
    B = small_batch(seed=4, n=8)
    v, f, r = to_dev(B)
    tb = TriangleBatch()
    for _ in range(3):
        tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"])
    # a different ray count per scene drops the graph and stays correct
    ro = B["ray_offsets"].copy()
    ro[1:] -= np.arange(1, ro.size, dtype=np.uint64)  # one ray fewer per scene
    keep = np.concatenate([np.arange(int(B["ray_offsets"][s]), int(B["ray_offsets"][s + 1]) - 1)
                           for s in range(ro.size - 1)])
    r2 = r[torch.as_tensor(keep).cuda()].contiguous()
    out = hits_np(tb.build_trace(v, f, B["face_offsets"], r2, ro))
    assert not tb.config()[2]
    B2 = dict(B, ray_offsets=ro)
    assert_same(out, per_scene(B2, v, f, r2))


def test_invalid_batches_are_rejected():
    B = small_batch(seed=5, n=3)
    v, f, r = to_dev(B)
    tb = TriangleBatch()
    fo, ro = B["face_offsets"], B["ray_offsets"]
    bad_fo = fo.copy()
    bad_fo[1] = 1  # a one-face scene
    with pytest.raises(sb.SurfaceError):
        tb.build_trace(v, f, bad_fo, r, ro)
    with pytest.raises(sb.SurfaceError):
        tb.build_trace(v, f, fo + 1, r, ro)  # offsets must start at 0
    with pytest.raises(sb.SurfaceError):
        tb.build_trace(v, f, fo[:2], r, ro)  # lengths differ


def test_full_size_batch_matches_per_scene():
    """64 scenes, 1e3-1e6 faces, images 128^2..1024^2: the batch against the
    per-scene GPU loop and every scene against the oracle."""
    B = S.batched_scenes()
    v, f, r = to_dev(B)
    tb = TriangleBatch()
    h = hits_np(tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"]))
    torch.cuda.synchronize()
    assert_same(h, per_scene(B, v, f, r))
    for _ in range(2):  # capture, then replay
        tb.build_trace(v, f, B["face_offsets"], r, B["ray_offsets"], hits=tb._keep[3])
    assert tb.config()[2]
    assert_same(hits_np(tb._keep[3]), h)
    # every scene against the oracle (its own build and trace of the scene)
    fo, ro = B["face_offsets"], B["ray_offsets"]
    for s_ in range(fo.size - 1):
        faces = B["faces"][int(fo[s_]):int(fo[s_ + 1])]
        o = O.OracleAccel(O.TRI, B["vertices"], faces)
        want = o.trace(B["rays"][int(ro[s_]):int(ro[s_ + 1])])
        assert_same(h[int(ro[s_]):int(ro[s_ + 1])], want)
