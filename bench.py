"""Benchmark: LBVH build + closest-hit throughput on B200 (one JSON line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tet|tri|particles|volume|volume_nu|batched|frame|scene|texture|lines|solids]

Default workload (``tri``): the plain triangle configuration -- an octasphere
of 131,072 FP32 triangles displaced radially by seeded value noise, 512x512
pinhole rays from distance 3 (45 deg).  One step = LBVH build from the
resident mesh + closest hit (prim, t, u, v) for every ray.  ``value`` = rays
per second of the whole step (build included), in Mrays/s.  ``tet`` is the
tetrahedral-mesh configuration (64^3 cells x 5 = 1,310,720 tets, FP64
Pluecker test, 1024^2 orthographic rays, barycentric scalar); ``particles``
one frame of the 16,777,216-sphere configuration (rebuild + 2048^2
primaries); ``texture`` 16,777,216 texture3D fetches of a 512^3 sparse byte
volume, in Mfetches/s.

Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events
on the launching stream; the L2 is flushed (256 MiB write) between steps,
outside the events.  Multi-GPU (torchrun): every rank runs the same workload
(independent replicas, weak scaling); the step time is the max over ranks.
``e2e`` repeats the step through the C ABI with pinned host buffers (mesh and
rays copied in, hits and scalars copied out every step).

``--impl reference`` times the reference's own CPU code (Build32 + OpenMP
Traverse, compiled from its sources into oracle/_ref) on the host cores, for
every ray of the step (nothing sampled or scaled).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def peaks():
    try:
        with open(MEASURED) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return FALLBACK_HBM, "fallback"


# ---------------------------------------------------------------- workloads
def make_workload(name):
    from surface_b200 import scenes as S
    if name == "tet":
        v, f, sc = S.tet_grid(64)
        rays = S.ortho_rays(1024, 1024)
        return dict(kind="tet", verts=v, prims=f, scalar=sc, rays=rays,
                    config={"workload": "tet64: 1,310,720 tetrahedra (64^3 cells x 5), "
                                        "1024x1024 orthographic rays, closest hit + "
                                        "barycentric scalar",
                            "prims": int(f.shape[0]), "rays": int(rays.size)})
    if name == "tri":
        v, f = S.displaced_octasphere(7)
        rays = S.pinhole_rays(512, 512, (0, 0, 3), (0, 0, 0))
        return dict(kind="tri", verts=v, prims=f, rays=rays,
                    config={"workload": "tri131k: displaced octasphere, 131,072 triangles, "
                                        "512x512 pinhole rays",
                            "prims": int(f.shape[0]), "rays": int(rays.size)})
    if name == "particles":
        pos, rad = S.particles()
        rays = S.pinhole_rays(2048, 2048, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
        return dict(kind="sphere", verts=pos, radius=rad, rays=rays, frames=10,
                    config={"workload": "particles16M: 16,777,216 spheres advected over 10 "
                                        "frames (step k = frame k mod 10): LBVH rebuild, "
                                        "2048x2048 pinhole primaries, one uniform-hemisphere "
                                        "secondary per hit with the self-hit rule",
                            "prims": int(pos.shape[0]), "primary_rays": int(rays.size),
                            "frames": 10})
    if name == "volume":
        dens = S.volume_blobs(256, nblobs=32)
        tgt = S.volume_blobs(256, nblobs=32, shift_voxels=2.0)
        tf = S.transfer_function(256)
        return dict(kind="volume", dens=dens, target_dens=tgt, tf=tf,
                    rays=np.zeros(512 * 512, np.uint8),
                    config={"workload": "volume256: 256^3 FP32 density (32 Gaussian blobs), "
                                        "256-entry RGBA transfer function, 512x512 rays, "
                                        "step 0.5 voxel, emission-absorption forward + "
                                        "adjoint of an L2 loss",
                            "rays": 512 * 512})
    if name == "volume_nu":
        W = make_workload("volume")
        W["nonuniform"] = True
        W["config"] = {"workload": "volume256-nu: the volume256 march with the y axis "
                                   "remapped through a 257-entry exponential coordinate "
                                   "table and GL's repeat wrap (the reference's non-uniform "
                                   "volume example), forward + adjoint",
                       "rays": 512 * 512}
        return W
    if name == "frame":
        v, f = S.displaced_octasphere(7)
        return dict(kind="frame", verts=v, prims=f, rays=np.zeros(512 * 512, np.uint8),
                    cam=dict(width=512, height=512, eye=(0.0, 0.0, 3.0),
                             lookat=(0.0, 0.0, 0.0), fov=45.0),
                    config={"workload": "frame512: tri131k scene (built once, resident), "
                                        "512x512 pinhole camera at distance 3, 45 deg: eye "
                                        "rays + closest hit + RGBA8 and depth write per step",
                            "prims": int(f.shape[0]), "rays": 512 * 512})
    if name == "scene":
        E = S.instanced_scene()
        return dict(kind="scene", E=E, rays=np.zeros(1024 * 1024, np.uint8),
                    cam=dict(width=1024, height=1024, eye=(-14.0, 10.0, 18.0),
                             lookat=(0.0, 0.0, 0.0), fov=40.0),
                    config={"workload": "scene64: 64 transformed elements on a 4x4x4 grid "
                                        "(instances of a 131,072-triangle octasphere, a "
                                        "1,000,000-sphere cloud and a 163,840-tet grid; "
                                        "accels resident), 1024x1024 pinhole camera: "
                                        "top-level tree build + eye rays + scene closest "
                                        "hit + RGBA8 and depth write per step",
                            "elements": len(E["elements"]),
                            "prims": int(sum(E["prims"])), "rays": 1024 * 1024})
    if name == "solids":
        v, ix = S.solid_grid(8, 64, seed=123456)
        rays = S.pinhole_rays(512, 512, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)
        return dict(kind="solids", verts=v, prims=ix, rays=rays,
                    config={"workload": "hex64: 262,144 hexahedra (64^3 jittered cells), "
                                        "512x512 pinhole rays; SolidAccel Build32 + closest "
                                        "hit with position and normal per step",
                            "prims": int(ix.shape[0]), "rays": int(rays.size)})
    if name == "lines":
        pos, seg, rad = S.line_strands(100000, 16, seed=123456)
        rays = S.pinhole_rays(1024, 1024, (0.3, 0.5, 3.4), (0, 0, 0), fov_deg=40)
        return dict(kind="lines", pos=pos, seg=seg, rad=rad, rays=rays,
                    config={"workload": "hair1.6M: 100,000 strands x 16 capped cylinders "
                                        "(1,600,000 lines, tapered radius 0.004) on the "
                                        "unit sphere, 1024x1024 pinhole rays; closest hit "
                                        "+ normal per step, accel resident (built once)",
                            "lines": int(seg.shape[0]), "rays": int(rays.size)})
    if name == "texture":
        blocks, pool, gdim = S.sparse_pages()
        uvw = S.march_coords()
        return dict(kind="texture", blocks=blocks, pool=pool, gdim=gdim, uvw=uvw,
                    rays=np.zeros(uvw.shape[0], np.uint8),
                    config={"workload": "sparse512: 512^3 sparse volume of 32^3 byte pages "
                                        "in a 3D checkerboard (2048 of 4096 committed), "
                                        "16,777,216 texture3D fetches per step (512x512 "
                                        "march rays x 64 samples, ray-major)",
                            "blocks": int(blocks.size), "fetches": int(uvw.shape[0])})
    if name == "batched":
        B = S.batched_scenes()
        return dict(kind="batched", B=B, rays=B["rays"],
                    config={"workload": "batched64: 64 displaced-octasphere triangle scenes, "
                                        "faces log-uniform in [1e3,1e6] (>= 1024), square "
                                        "pinhole images of side 128/256/512/1024",
                            "scenes": 64, "prims": int(B["face_offsets"][-1]),
                            "rays": int(B["ray_offsets"][-1])})
    raise SystemExit(f"unknown workload {name}")


# build: vertices of each triangle (3 x 12) read twice (bbox, Morton) and once
# more in the refit, code + index written and read per radix pass (5 passes
# x 16), leaf record (48) written, internal node (64) written, Karras tree
# arrays (~40 per node) written and read
BUILD_BYTES_PER_TRI = 3 * 36 + 5 * 16 + 48 + 64 + 40


PROFILES = os.path.join(ROOT, "profiles")
# DRAM bytes per launch of the dominant kernel, from the committed ncu capture
TRAFFIC_PROFILE = {"tet": "trace_tet_kernel.tet64.md"}


def profiled_traffic(kind):
    try:
        with open(os.path.join(PROFILES, TRAFFIC_PROFILE[kind])) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":")[1])
    except Exception:  # noqa: BLE001
        pass
    return None


def algorithmic_bytes_per_ray(kind, stats, nrays):
    """Per-ray bytes the traversal must move: ray (32) + hit (16) + nodes
    visited x node size + primitives tested x primitive record."""
    branch, leaf, prim = (float(x) / nrays for x in stats)
    if kind == "tet":
        return 32 + 16 + 4 + 4 + branch * 32 + prim * (48 + 4)
    if kind == "tri":
        return 32 + 16 + branch * 64 + prim * 48
    return 32 + 16 + branch * 64 + prim * (16 + 4)


# ---------------------------------------------------------------- clocks
def e2e_warmup(step, args, min_steps=10, min_s=0.25):
    """Untimed end-to-end steps before the timed ones: at least the bench's
    warm-up count, `min_steps` and `min_s` seconds -- the first host-driven
    steps after the device-timed loop run well above the steady state (host
    allocations and the clock sampler's exit just before them)."""
    t_end = time.perf_counter() + min_s
    k = 0
    while k < max(args.warmup, 3, min_steps) or time.perf_counter() < t_end:
        step()
        k += 1


class ClockSampler:
    def __init__(self, device):
        self.proc = None
        self.device = device
        self.first = None
        self.path = os.path.join("/tmp", f"srt_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()
        try:
            self.f.close()
        except Exception:  # noqa: BLE001
            pass

    def count(self):
        try:
            self.f.flush()
            with open(self.path) as f:
                return sum(1 for line in f if line.strip())
        except Exception:  # noqa: BLE001
            return 0

    def keep_busy(self, step, sync, extra=2, limit_s=3.0):
        """Run `step` until `extra` more clock samples have landed (the
        sampler starts slower than a short timed region), bounded in time."""
        if self.proc is None:
            return
        n0 = self.count()
        if self.first is None:
            self.first = n0  # samples before the first busy period are idle
        t_end = time.time() + limit_s
        while self.count() < n0 + extra and time.time() < t_end:
            step()
            sync()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
            rows = rows[self.first or 0:] or rows
            sm = [float(r[0]) for r in rows if r[0].strip().isdigit()]
            mx = max(float(r[1]) for r in rows)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[k] for r in rows for k in range(4)
                              if r[3 + k].strip() == "Active"})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                    "reasons": reasons, "samples": len(rows)}
        except Exception:  # noqa: BLE001
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


# ---------------------------------------------------------------- ranks
def dist_setup(dev):
    """One process per GPU (torchrun): NCCL on CUDA, gloo on CPU; returns
    (world, rank).  The group only carries the barrier and the max-over-ranks
    step time: replicas exchange no data."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        kw = {"device_id": dev} if dev.type == "cuda" else {}
        dist.init_process_group("nccl" if dev.type == "cuda" else "gloo",
                                timeout=datetime.timedelta(seconds=120), **kw)
    return world, rank


def _dist_on():
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier():
    if _dist_on():
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(vals, dev):
    """Element-wise maximum of per-rank values (step times) over all ranks."""
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=dev)
    if _dist_on():
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu().tolist()]


def whole_job_mrays(units_per_rank, world, ms_per_step):
    """Rays of all ranks per second of the slowest rank, in Mrays/s."""
    return world * units_per_rank / (ms_per_step * 1e-3) / 1e6


def dist_teardown():
    if _dist_on():
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- CPU side
def cpu_reference_step(W, nthreads=0, stride=1):
    """Reference Build32 + OpenMP Traverse of every ray (every stride-th ray
    when stride > 1, the trace time then scaled to all rays).
    Returns (Mrays/s, build s, trace s, rays traced, kind)."""
    from oracle import oracle as O
    kind = {"tet": O.TET, "tri": O.TRI, "sphere": O.SPHERE}[W["kind"]]
    use_ref = O.have_ref() and O.ref() is not None
    t0 = time.perf_counter()
    if use_ref:
        acc = O.RefAccel(kind, W["verts"], W.get("prims"), W.get("radius"))
    else:
        acc = O.OracleAccel(kind, W["verts"], W.get("prims"), W.get("radius"))
    tb = time.perf_counter() - t0
    sample = W["rays"][::stride]
    t0 = time.perf_counter()
    if use_ref:
        acc.trace(sample, nthreads=nthreads, chunk=64)
    else:
        acc.trace(sample, nthreads=nthreads)
    tt = time.perf_counter() - t0
    nr = W["rays"].size
    value = nr / (tb + tt * (nr / sample.size)) / 1e6
    return value, tb, tt, sample.size, ("reference" if use_ref else "port")


def cpu_reference_batched(W, nthreads=0, stride=1):
    """Reference loop over the scenes: Build32 of every scene + OpenMP
    Traverse of every ray of each (every stride-th ray when stride > 1,
    scaled).  Returns (Mrays/s, build s, trace s, rays traced, kind)."""
    from oracle import oracle as O
    B = W["B"]
    use_ref = O.have_ref() and O.ref() is not None
    fo, ro = B["face_offsets"], B["ray_offsets"]
    tb = tt = 0.0
    ns = 0
    for s in range(fo.size - 1):
        faces = B["faces"][int(fo[s]):int(fo[s + 1])]
        t0 = time.perf_counter()
        acc = (O.RefAccel if use_ref else O.OracleAccel)(O.TRI, B["vertices"], faces)
        tb += time.perf_counter() - t0
        sample = B["rays"][int(ro[s]):int(ro[s + 1])][::stride]
        t0 = time.perf_counter()
        if use_ref:
            acc.trace(sample, nthreads=nthreads, chunk=64)
        else:
            acc.trace(sample, nthreads=nthreads)
        tt += time.perf_counter() - t0
        ns += sample.size
        del acc
    nr = int(ro[-1])
    value = nr / (tb + tt * (nr / ns)) / 1e6
    return value, tb, tt, ns, ("reference" if use_ref else "port")


def cpu_reference_particles(W, nthreads=0, stride=1):
    """Reference Build32 of the frame-0 cloud + OpenMP Traverse of every
    primary and every secondary (every stride-th when stride > 1, scaled);
    the secondaries are spawned from the reference's own primary hits by the
    workload's bounce rule, outside the timed calls.  Returns (Mrays/s, build
    s, trace s, rays traced, kind)."""
    from oracle import oracle as O
    from surface_b200 import scenes as S
    use_ref = O.have_ref() and O.ref() is not None
    Acc = O.RefAccel if use_ref else O.OracleAccel
    t0 = time.perf_counter()
    acc = Acc(O.SPHERE, W["verts"], None, W["radius"])
    tb = time.perf_counter() - t0
    kw = {"nthreads": nthreads, "chunk": 64} if use_ref else {"nthreads": nthreads}
    prim = W["rays"]
    t0 = time.perf_counter()
    h1 = acc.trace(prim[::stride], **kw)
    tt = time.perf_counter() - t0
    nrm = S.sphere_normals_np(prim[::stride], h1, W["verts"])
    sec, sn = S.spawn_secondary_np(prim[::stride], h1, nrm, 0)
    t0 = time.perf_counter()
    acc.trace(sec, prev_normals=sn, **kw)
    tt += time.perf_counter() - t0
    ns = prim[::stride].size + sec.size
    total = stride * ns  # primaries + secondaries of the whole frame (scaled)
    value = total / (tb + tt * stride) / 1e6
    return value, tb, tt, ns, ("reference" if use_ref else "port")


def cpu_reference_frame(W, nthreads=0):
    """OnData on the host: the eye rays and framebuffer write of the CPU
    restatement around the reference's own OpenMP Traverse over every pixel
    (the accel is built once, outside the timing, as AccelBuilder caches it).
    Returns (Mrays/s, rays s, trace s, rays, kind)."""
    from oracle import oracle as O
    from surface_b200 import camera as K
    use_ref = O.have_ref() and O.ref() is not None
    if "_cpu_acc" not in W:
        W["_cpu_acc"] = (O.RefAccel if use_ref else O.OracleAccel)(O.TRI, W["verts"],
                                                                   W["prims"])
    acc = W["_cpu_acc"]
    d = K.camera_dict(K.make_camera(**W["cam"]))
    t0 = time.perf_counter()
    rays, pix = O.camera_rays(d)
    tr = time.perf_counter() - t0
    t0 = time.perf_counter()
    hits = acc.trace(rays, nthreads=nthreads, chunk=64) if use_ref else acc.trace(
        rays, nthreads=nthreads)
    tt = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.framebuffer_write(d, hits, pix, None, 0)
    tr += time.perf_counter() - t0
    return rays.size / (tr + tt) / 1e6, tr, tt, rays.size, ("reference" if use_ref else "port")


def _oracle_scene(W):
    from oracle import oracle as O
    if "_cpu_scene" not in W:
        E = W["E"]
        accs = []
        for a in E["accels"]:
            if a["kind"] == 2:
                accs.append(O.OracleAccel(O.SPHERE, a["verts"], None, a["radius"]))
            else:
                accs.append(O.OracleAccel(O.TRI if a["kind"] == 0 else O.TET, a["verts"],
                                          a["faces"]))
        W["_cpu_accs"] = accs
        W["_cpu_scene"] = None
    return W["_cpu_accs"]


def cpu_reference_scene(W, nthreads=0, stride=1):
    """The CPU restatement of one scene frame (RenderGraph::Build, the eye
    rays, RenderGraph::Trace with OpenMP over every pixel, the
    framebuffer write); element accels built once outside the timing.
    Returns (Mrays/s, build+rays+write s, trace s scaled, rays traced, kind)."""
    from oracle import oracle as O
    from surface_b200 import camera as K
    accs = _oracle_scene(W)
    E = W["E"]
    d = K.camera_dict(K.make_camera(**W["cam"]))
    t0 = time.perf_counter()
    mats = [O.element_update(el["T"], *accs[el["accel"]].bbox64())
            for el in E["elements"]]
    sc = O.OracleScene([accs[el["accel"]] for el in E["elements"]],
                       [el["T"] for el in E["elements"]], [m[0] for m in mats],
                       [m[1] for m in mats], [m[2] for m in mats], [m[3] for m in mats])
    rays, pix = O.camera_rays(d)
    tr = time.perf_counter() - t0
    sample = rays[::stride]
    t0 = time.perf_counter()
    hits, _ = sc.trace(sample, nthreads=nthreads)
    tt = (time.perf_counter() - t0) * stride
    t0 = time.perf_counter()
    O.framebuffer_write(d, hits, pix[::stride], None, 0)
    tr += (time.perf_counter() - t0)
    return rays.size / (tr + tt) / 1e6, tr, tt, sample.size, "port"


def cpu_reference_texture(W, nthreads=0):
    """Texture::Fetch of every coordinate on the host: the reference's own
    SparseVolumeAccel (oracle/_ref) or else the CPU restatement, over
    nthreads threads (each builds its block tree, as every texture unit of
    the reference would).  Returns (Mfetches/s, 0, s, fetches, kind)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    use_ref = O.have_ref() and O.ref() is not None
    nt = nthreads or os.cpu_count() or 1
    uvw = W["uvw"]
    parts = np.array_split(np.arange(uvw.shape[0]), nt)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(nt) as ex:
        list(ex.map(lambda ix: O.sparse_fetch(W["blocks"], W["pool"], 0, 1, W["gdim"],
                                              uvw[ix[0]:ix[-1] + 1], use_ref=use_ref),
                    [q for q in parts if q.size]))
    tt = time.perf_counter() - t0
    return (uvw.shape[0] / tt / 1e6, 0.0, tt, uvw.shape[0],
            "reference" if use_ref else "port")


def cpu_reference_solids(W, nthreads=0, stride=1):
    """SolidAccel::Build32 of the mesh and Traverse of every stride-th ray on
    the host: the reference's own code (oracle/_ref) or else the
    restatement, OpenMP over all cores.  Returns (Mrays/s, build s, trace s
    scaled, rays traced, kind)."""
    from oracle import oracle as O
    use_ref = O.have_ref() and O.ref() is not None
    t0 = time.perf_counter()
    acc = (O.RefSolids if use_ref else O.OracleSolids)(8, W["verts"], W["prims"])
    tb = time.perf_counter() - t0
    sample = W["rays"][::stride]
    t0 = time.perf_counter()
    acc.trace(sample, nthreads=nthreads)
    tt = (time.perf_counter() - t0) * stride
    return (W["rays"].size / (tb + tt) / 1e6, tb, tt, sample.size,
            "reference" if use_ref else "port")


def cpu_reference_lines(W, nthreads=0, stride=1):
    """LineAccel::Traverse of every stride-th ray on the host: the
    reference's own code (oracle/_ref) or else the restatement, OpenMP over
    all cores; the accel is built once outside the timing.  Returns
    (Mrays/s, build s, trace s scaled, rays traced, kind)."""
    from oracle import oracle as O
    use_ref = O.have_ref() and O.ref() is not None
    if "_cpu_lines" not in W:
        t0 = time.perf_counter()
        W["_cpu_lines"] = (O.RefLines if use_ref else O.OracleLines)(W["pos"], W["seg"],
                                                                      W["rad"])
        W["_cpu_lines_build"] = time.perf_counter() - t0
    acc = W["_cpu_lines"]
    sample = W["rays"][::stride]
    t0 = time.perf_counter()
    acc.trace(sample, nthreads=nthreads)
    tt = (time.perf_counter() - t0) * stride
    return (W["rays"].size / tt / 1e6, W["_cpu_lines_build"], tt, sample.size,
            "reference" if use_ref else "port")


def run_reference_arm(args, W):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    step = {"batched": cpu_reference_batched, "sphere": cpu_reference_particles,
            "frame": cpu_reference_frame, "scene": cpu_reference_scene,
            "texture": cpu_reference_texture, "lines": cpu_reference_lines,
            "solids": cpu_reference_solids}.get(W["kind"], cpu_reference_step)
    for _ in range(args.warmup):
        step(W)
    vals, tbs, tts = [], [], []
    flush = np.zeros(256 * 1024 * 1024 // 8, np.float64)
    for _ in range(args.steps):
        flush[:] = 1.0  # 256 MiB written between steps: host caches hold no step state
        v, tb, tt, ns, kind = step(W)
        vals.append(v)
        tbs.append(tb)
        tts.append(tt)
    value = statistics.median(vals)
    # every ray is traced (no scaling): the median step's measured time
    ms = 1e3 * ns / (value * 1e6)
    unit = "Mfetches/s" if W["kind"] == "texture" else "Mrays/s"
    sample = (f"the full step: Build32 + Traverse of every ray ({ns}) through the "
              f"reference's own code (OpenMP, {cores} threads); median of {args.steps}")
    if W["kind"] == "batched":
        sample = (f"the full step: Build32 + Traverse of every ray of all 64 scenes ({ns}) "
                  f"through the reference's own code (OpenMP, {cores} threads); median of "
                  f"{args.steps}")
    if W["kind"] == "sphere":
        sample = (f"the full frame: Build32 + Traverse of every primary and every "
                  f"secondary ({ns} rays) through the reference's own code (OpenMP, "
                  f"{cores} threads); median of {args.steps}")
    if W["kind"] == "frame":
        sample = (f"every pixel ({ns} rays): eye rays and framebuffer write of the CPU "
                  f"restatement, Traverse of the reference (accel built once); median of "
                  f"{args.steps}")
    if W["kind"] == "scene":
        sample = (f"top-level build, eye rays, scene trace and write of every pixel ({ns}) "
                  f"by the CPU restatement (OpenMP; the reference's RenderGraph needs its "
                  f"GL front end); median of {args.steps}")
    if W["kind"] == "solids":
        sample = (f"full Build32 + Traverse of every ray ({ns}) per step through the "
                  f"reference's own SolidAccel (OpenMP, {cores} threads); median of "
                  f"{args.steps}")
    if W["kind"] == "lines":
        sample = (f"every ray ({ns}) per step through the reference's own "
                  f"LineAccel::Traverse (OpenMP, {cores} threads; accel built once); "
                  f"median of {args.steps}")
    if W["kind"] == "texture":
        sample = (f"every fetch ({ns}) per step through the reference's own "
                  f"SparseVolumeAccel (Build + Sample) over {cores} threads; median of "
                  f"{args.steps}")
    line = {
        "impl": "reference",
        "metric": {"batched": METRIC_BATCH, "sphere": METRIC_PART,
                   "frame": METRIC_FRAME, "scene": METRIC_SCENE,
                   "texture": METRIC_TEX, "lines": METRIC_LINES,
                   "solids": METRIC_SOLIDS}.get(W["kind"], METRIC),
        "value": round(value, 4), "unit": unit,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE[W["kind"]], "data": "synthetic",
        "config": dict(W["config"], l2="flushed between steps (256 MiB write)",
                       parallelism=f"replicas x{args.gpus}"),
        ("rays_write_ms" if W["kind"] in ("frame", "scene") else "build_ms"):
            round(1e3 * statistics.median(tbs), 3),
        "cpu_baseline": {"value": round(value, 4), "unit": unit, "cores": cores,
                         "kind": kind, "sample": sample},
        "e2e": {"value": round(value, 4), "unit": unit, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if W["kind"] == "texture":
        line.pop("build_ms", None)
    print(json.dumps(line), flush=True)


METRIC = "Mrays/s (LBVH build + closest hit per step)"
METRIC_VOL = "Mrays/s (volume march forward + adjoint per step)"
METRIC_BATCH = "Mrays/s (64-scene batched LBVH build + closest hit per step)"
METRIC_PART = "Mrays/s (particle frame: LBVH rebuild + primaries + secondaries per step)"
METRIC_FRAME = "Mrays/s (frame: eye rays + closest hit + framebuffer write per step)"
METRIC_SCENE = ("Mrays/s (scene frame: top-level build + eye rays + closest hit over "
                "transformed elements + framebuffer write per step)")
METRIC_TEX = "Mfetches/s (sparse volume texture3D fetch per step)"
METRIC_LINES = "Mrays/s (capped-cylinder line accel: closest hit + normal per step)"
METRIC_SOLIDS = "Mrays/s (hexahedron solid accel: Build32 + closest hit per step)"
DTYPE = {"tet": "f32 boxes / f64 Pluecker", "tri": "f32", "sphere": "f32 (f64 discriminant)",
         "texture": "u8 texels / f64 block tree",
         "lines": "f32 (f64 quadratic root)",
         "solids": "f32 boxes / f64 Pluecker",
         "volume": "f32", "batched": "f32", "frame": "f32",
         "scene": "f64 transforms and top-level boxes / f32 + f64 element tests"}


def volume_sample_count(p):
    """Samples the march takes: floor((t1 - t0) / step) per pixel ray through
    the [-1, 1]^3 slab (the kernel's camera and slab test, in float64)."""
    W, H = int(p["width"][0]), int(p["height"][0])
    px, py = np.meshgrid(np.arange(W) + 0.5, np.arange(H) + 0.5)
    v = (p["corner"][0][None, None, :] + px[..., None] * p["du"][0] + py[..., None] * p["dv"][0]
         - p["eye"][0])
    d = v / np.linalg.norm(v, axis=-1, keepdims=True)
    o = p["eye"][0].astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        tn = (-1.0 - o) / d
        tf = (1.0 - o) / d
    t0 = np.maximum(np.minimum(tn, tf).max(-1), -10000.0)
    t1 = np.minimum(np.maximum(tn, tf).min(-1), 10000.0)
    ns = np.where(t0 <= t1, np.floor((t1 - t0) / float(p["step"][0])), 0)
    return float(np.minimum(ns, int(p["max_steps"][0])).sum())


def run_volume(args, W):
    """Forward + adjoint of the L2 loss per step (device resident); forward
    alone is timed too.  CPU baseline: the FP32 oracle forward (OpenMP)."""
    import torch

    from surface_b200 import volume as V
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    p = V.camera(512, 512, res=256)
    dens = torch.as_tensor(W["dens"], device=dev)
    tf = torch.as_tensor(W["tf"], device=dev)
    smp = None
    if W.get("nonuniform"):
        from surface_b200 import scenes as S
        smp = V.Sampling(remap=(None, S.exp_coord_map(257), None), clamp=(False,) * 3,
                         device=dev.index)
    target = V.march(torch.as_tensor(W["target_dens"], device=dev), tf, p, sampling=smp)[0]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def fwd():
        return V.march(dens, tf, p, sampling=smp)

    def fwd_bwd():
        img, tr = V.march(dens, tf, p, sampling=smp)
        return V.march_backward(dens, tf, p, tr, 2 * (img - target), sampling=smp)

    from surface_b200 import _lib
    from surface_b200.accel import Context
    L = _lib.load()
    vctx = Context.default(dev.index)
    for _ in range(max(args.warmup, 3)):
        fwd_bwd()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    fe = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(dev.index) as clk:
        clk.keep_busy(fwd_bwd, torch.cuda.synchronize)
        launches0 = L.srt_ctx_launch_count(vctx.h)
        for k in range(args.steps):
            flush.zero_()
            fe[k][0].record()
            fwd()
            fe[k][1].record()
            flush.zero_()
            ev[k][0].record()
            fwd_bwd()
            ev[k][1].record()
        torch.cuda.synchronize()
        launches = L.srt_ctx_launch_count(vctx.h) - launches0
        clk.keep_busy(fwd_bwd, torch.cuda.synchronize, extra=1)
    fb_ms, f_ms = max_over_ranks([statistics.mean(a.elapsed_time(b) for a, b in ev),
                                  statistics.mean(a.elapsed_time(b) for a, b in fe)], dev)
    nr = 512 * 512

    # ---- e2e: density and table copied in from pinned host memory, both
    # gradients copied back, every step
    h_dens = torch.from_numpy(np.ascontiguousarray(W["dens"])).pin_memory()
    h_tf = torch.from_numpy(np.ascontiguousarray(W["tf"])).pin_memory()
    h_gd = torch.empty_like(h_dens).pin_memory()
    h_gt = torch.empty_like(h_tf).pin_memory()

    def e2e_step():
        dens.copy_(h_dens, non_blocking=True)
        tf.copy_(h_tf, non_blocking=True)
        gd, gt = fwd_bwd()
        h_gd.copy_(gd, non_blocking=True)
        h_gt.copy_(gt, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]
    e2e = {"value": round(whole_job_mrays(nr, world, e2e_ms), 3), "unit": "Mrays/s",
           "h2d_bytes_per_step": int((h_dens.numel() + h_tf.numel()) * 4),
           "d2h_bytes_per_step": int((h_gd.numel() + h_gt.numel()) * 4),
           "ms_per_step": round(e2e_ms, 3)}

    # ---- roofline of the adjoint kernel (the larger of the two): unique
    # bytes it must move -- density read, density gradient written, image-
    # sized inputs -- against HBM; the samples' trilinear gathers (32 B each)
    # are served by L1/L2 and reported beside it
    hbm, src = peaks()
    nsamp = volume_sample_count(p)
    bwd_ms = fb_ms - f_ms
    uniq = 2 * W["dens"].nbytes + nr * (16 + 4 + 16) + 2 * W["tf"].nbytes
    roofline = {"bound": "hbm", "kernel": "vol_bwd_kernel (fwd+bwd minus fwd)",
                "achieved": round(uniq / (bwd_ms * 1e-3) / 1e9, 1), "peak": hbm,
                "unit": "GB/s", "frac": round(uniq / (bwd_ms * 1e-3) / 1e9 / hbm, 4),
                "peak_source": src, "traffic": None,
                "algorithmic_bytes_per_launch": int(uniq), "samples": int(nsamp),
                "sample_gather_gbs": round(32 * nsamp / (bwd_ms * 1e-3) / 1e9, 1)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        q = np.zeros(1, O.VOL_DTYPE)
        q[...] = p.view(O.VOL_DTYPE)
        t0 = time.perf_counter()
        if W.get("nonuniform"):
            from surface_b200 import scenes as S
            O.volume_fwd_f32(q, W["dens"], (256, 256, 256), W["tf"],
                             remap=(None, S.exp_coord_map(257), None), clamp=(0, 0, 0))
        else:
            O.volume_fwd_f32(q, W["dens"], (256, 256, 256), W["tf"])
        tc = time.perf_counter() - t0
        cpu = {"value": round(nr / tc / 1e6, 4), "unit": "Mrays/s", "cores": os.cpu_count(),
               "kind": "port", "sample": "FP32 forward march restatement over all 512^2 "
                                         "rays (the reference has no C++ march; its shader "
                                         "march needs the closed GLSL compiler)",
               "forward_ms": round(1e3 * tc, 2)}
    line = {"metric": METRIC_VOL, "value": round(whole_job_mrays(nr, world, fb_ms), 3),
            "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(fb_ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)"),
            "forward_ms": round(f_ms, 4), "forward_backward_ms": round(fb_ms, 4),
            "fwd_bwd_over_fwd": round(fb_ms / f_ms, 3), "clocks": clk.summary(),
            "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline,
            "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(line), flush=True)
    dist_teardown()


# ---------------------------------------------------------------- texture
# algorithmic bytes of one sparse fetch: its coordinate (12) read, its RGBA
# (16) written, one byte texel read (the block tree, 4095 nodes, stays cached)
TEX_BYTES_PER_FETCH = 12 + 16 + 1


def run_texture(args, W):
    """Texture::Fetch of a sparse volume: every step fetches all coordinates
    (device resident, larger than L2).  e2e: coordinates from pinned host
    memory in, RGBA back, every step."""
    import torch

    from surface_b200 import _lib
    from surface_b200.texture import Texture3D
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    tex = Texture3D(device=dev.index)
    tex.set_sparse(W["blocks"], W["pool"], 0, 1, W["gdim"])
    L = _lib.load()
    n = W["uvw"].shape[0]
    uvw = torch.as_tensor(W["uvw"], device=dev)
    out = torch.empty((n, 4), dtype=torch.float32, device=dev)

    def step():
        tex.Fetch(uvw, out)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(dev.index) as clk:
        clk.keep_busy(step, torch.cuda.synchronize)
        barrier()
        torch.cuda.synchronize()
        launches0 = L.srt_ctx_launch_count(tex.ctx.h)
        for k in range(args.steps):
            ev[k][0].record()
            step()
            ev[k][1].record()
        torch.cuda.synchronize()
        barrier()
        launches = L.srt_ctx_launch_count(tex.ctx.h) - launches0
        clk.keep_busy(step, torch.cuda.synchronize, extra=1)
    ms = max_over_ranks([statistics.mean(a.elapsed_time(b) for a, b in ev)], dev)[0]
    value = world * n / (ms * 1e-3) / 1e6

    # e2e through the public call with host buffers
    h_uvw = torch.from_numpy(W["uvw"]).pin_memory()
    h_out = torch.empty((n, 4), dtype=torch.float32).pin_memory()

    def e2e_step():
        uvw.copy_(h_uvw, non_blocking=True)
        tex.Fetch(uvw, out)
        h_out.copy_(out, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]
    e2e = {"value": round(world * n / (e2e_ms * 1e-3) / 1e6, 3), "unit": "Mfetches/s",
           "h2d_bytes_per_step": int(h_uvw.numel() * 4),
           "d2h_bytes_per_step": int(h_out.numel() * 4), "ms_per_step": round(e2e_ms, 3)}
    # parity of this run's output with the restatement on a slice
    got = out[:65536].cpu().numpy()
    hbm, src = peaks()
    alg = TEX_BYTES_PER_FETCH * n
    traffic = None
    prof = os.path.join(PROFILES, "sparse_fetch_kernel.sparse512.md")
    if os.path.exists(prof):
        m = re.search(r"traffic_per_launch_bytes:\s*(\d+)", open(prof).read())
        traffic = int(m.group(1)) if m else None
    roofline = {"bound": "hbm", "kernel": "sparse_fetch_kernel",
                "achieved": round(alg / (ms * 1e-3) / 1e9, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(alg / (ms * 1e-3) / 1e9 / hbm, 4), "peak_source": src,
                "traffic": traffic, "algorithmic_bytes_per_launch": int(alg)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        want = O.sparse_fetch(W["blocks"], W["pool"], 0, 1, W["gdim"], W["uvw"][:65536])
        if not np.array_equal(got.view(np.uint32), want.view(np.uint32)):
            raise SystemExit("sparse fetch differs from the oracle")
        v, _, tt, ns, kind = cpu_reference_texture(W)
        cpu = {"value": round(v, 3), "unit": "Mfetches/s", "cores": os.cpu_count(),
               "kind": kind, "sample": f"all {ns} fetches, {os.cpu_count()} threads",
               "seconds": round(tt, 3)}
    line = {"metric": METRIC_TEX, "value": round(value, 3), "unit": "Mfetches/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE["texture"], "data": "synthetic",
            "config": dict(W["config"], l2="inputs larger than L2 (201 MB coordinates, "
                                           "268 MB RGBA)"),
            "clocks": clk.summary(), "e2e": e2e, "gpu_launches": int(launches),
            "roofline": roofline, "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(line), flush=True)
    tex.close()
    dist_teardown()


# ---------------------------------------------------------------- lines
def run_lines(args, W):
    """Closest hit + normal for every ray against the resident line accel
    (device rays, hits and normals larger than L2).  e2e: rays from pinned
    host memory in, hits and normals back, every step.  The GPU build (host
    input arrays in, the call returns when the tree is done) is timed over
    three calls after a first one, and again from device-resident inputs,
    and reported beside the line."""
    import torch

    from surface_b200 import _lib
    from surface_b200.lines import LineAccel, Lines
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    acc = LineAccel(device=dev.index)
    lines_in = Lines(W["pos"], W["seg"], W["rad"])
    acc.Build(lines_in)
    torch.cuda.synchronize()
    build_s = []
    for _ in range(3):
        t0 = time.perf_counter()
        acc.Build(lines_in)
        build_s.append(time.perf_counter() - t0)
    build_s = statistics.mean(build_s)
    # the same build from device-resident inputs (no staging copies)
    lines_dev = Lines(torch.as_tensor(W["pos"], device=dev),
                      torch.as_tensor(W["seg"].astype(np.int32), device=dev),
                      torch.as_tensor(W["rad"], device=dev))
    acc.Build(lines_dev)
    torch.cuda.synchronize()
    build_dev_s = []
    for _ in range(3):
        t0 = time.perf_counter()
        acc.Build(lines_dev)
        build_dev_s.append(time.perf_counter() - t0)
    build_dev_s = statistics.mean(build_dev_s)
    L = _lib.load()
    rays_np = W["rays"]
    n = rays_np.size
    rays = torch.from_numpy(rays_np.view(np.float32).reshape(-1, 8)).to(dev)
    hits = torch.empty((n, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty((n, 3), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def step():
        acc.ctx.use_torch_stream()
        check_line(L, acc, rays, n, hits, nrm)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(dev.index) as clk:
        clk.keep_busy(step, torch.cuda.synchronize)
        barrier()
        torch.cuda.synchronize()
        launches0 = L.srt_ctx_launch_count(acc.ctx.h)
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            step()
            ev[k][1].record()
        torch.cuda.synchronize()
        barrier()
        launches = L.srt_ctx_launch_count(acc.ctx.h) - launches0
        clk.keep_busy(step, torch.cuda.synchronize, extra=1)
    ms = max_over_ranks([statistics.mean(a.elapsed_time(b) for a, b in ev)], dev)[0]
    value = whole_job_mrays(n, world, ms)
    # work counters of one untimed pass: the bytes a ray touches
    stats = torch.zeros(3, dtype=torch.int64, device=dev)
    acc.Traverse(rays, hits, stats=stats)
    torch.cuda.synchronize()
    nb, nl, nt = (int(x) for x in stats.cpu())

    h_rays = torch.from_numpy(rays_np.view(np.float32).reshape(-1, 8).copy()).pin_memory()
    h_hits = torch.empty((n, 4), dtype=torch.float32).pin_memory()
    h_nrm = torch.empty((n, 3), dtype=torch.float32).pin_memory()

    def e2e_step():
        rays.copy_(h_rays, non_blocking=True)
        step()
        h_hits.copy_(hits, non_blocking=True)
        h_nrm.copy_(nrm, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]
    e2e = {"value": round(whole_job_mrays(n, world, e2e_ms), 3), "unit": "Mrays/s",
           "h2d_bytes_per_step": int(h_rays.numel() * 4),
           "d2h_bytes_per_step": int((h_hits.numel() + h_nrm.numel()) * 4),
           "ms_per_step": round(e2e_ms, 3)}
    # roofline: ray (32) + hit (16) + normal (12) per ray, 32 per branch
    # popped, 32 per leaf popped and 64 per line tested
    hbm, src = peaks()
    alg = n * (32 + 16 + 12) + 32 * (nb + nl) + 64 * nt
    traffic = None
    prof = os.path.join(PROFILES, "line_trace_kernel.hair1.6M.md")
    if os.path.exists(prof):
        m = re.search(r"traffic_per_launch_bytes:\s*(\d+)", open(prof).read())
        traffic = int(m.group(1)) if m else None
    roofline = {"bound": "hbm", "kernel": "line_trace_kernel",
                "achieved": round(alg / (ms * 1e-3) / 1e9, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(alg / (ms * 1e-3) / 1e9 / hbm, 4), "peak_source": src,
                "traffic": traffic, "algorithmic_bytes_per_launch": int(alg),
                "per_ray": {"branches": round(nb / n, 2), "leaves": round(nl / n, 2),
                            "line_tests": round(nt / n, 2)},
                "note": "node and line bytes are served mostly from L2 (tree 180 MB)"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        got = hits.cpu().numpy()[:: 97]
        want, _ = O.OracleLines(W["pos"], W["seg"], W["rad"]).trace(rays_np[:: 97])
        if not np.array_equal(got.view(np.uint32), want.view(np.float32).reshape(-1, 4)
                              .view(np.uint32)):
            raise SystemExit("line hits differ from the oracle")
        v, _, tt, ns, kind = cpu_reference_lines(W)
        cpu = {"value": round(v, 3), "unit": "Mrays/s", "cores": os.cpu_count(),
               "kind": kind, "sample": f"every ray ({ns}), OpenMP over "
                                       f"{os.cpu_count()} threads",
               "seconds": round(tt, 3)}
    line = {"metric": METRIC_LINES, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE["lines"], "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)"),
            "build_ms": round(1e3 * build_s, 2),
            "build_ms_device_inputs": round(1e3 * build_dev_s, 2), "clocks": clk.summary(), "e2e": e2e,
            "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(line), flush=True)
    acc.close()
    dist_teardown()


# ---------------------------------------------------------------- solids
def run_solids(args, W):
    """Build32 of the resident mesh + closest hit (position and normal) of
    every ray per step.  e2e: mesh and rays from pinned host memory in, hits
    back, every step."""
    import torch

    from surface_b200 import _lib
    from surface_b200.solids import Solid, SolidAccel
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    L = _lib.load()
    acc = SolidAccel(device=dev.index)
    v = torch.as_tensor(W["verts"], device=dev)
    ix = torch.as_tensor(W["prims"].astype(np.int32), device=dev)
    rays_np = W["rays"]
    n = rays_np.size
    rays = torch.from_numpy(rays_np.view(np.float32).reshape(-1, 8)).to(dev)
    hits = torch.empty((n, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty((n, 3), dtype=torch.float32, device=dev)
    pos = torch.empty((n, 3), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    from surface_b200._lib import check

    def step():
        acc.Build32(Solid(8, v, ix))
        acc.ctx.use_torch_stream()
        check(L.srt_solid_trace(acc.h, rays.data_ptr(), n, hits.data_ptr(), nrm.data_ptr(),
                                pos.data_ptr()))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    tev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(dev.index) as clk:
        clk.keep_busy(step, torch.cuda.synchronize)
        barrier()
        torch.cuda.synchronize()
        launches0 = L.srt_ctx_launch_count(acc.ctx.h)
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            acc.Build32(Solid(8, v, ix))
            acc.ctx.use_torch_stream()
            tev[k][0].record()
            check(L.srt_solid_trace(acc.h, rays.data_ptr(), n, hits.data_ptr(),
                                    nrm.data_ptr(), pos.data_ptr()))
            tev[k][1].record()
            ev[k][1].record()
        torch.cuda.synchronize()
        barrier()
        launches = L.srt_ctx_launch_count(acc.ctx.h) - launches0
        clk.keep_busy(step, torch.cuda.synchronize, extra=1)
    ms, tms = max_over_ranks([statistics.mean(a.elapsed_time(b) for a, b in ev),
                              statistics.mean(a.elapsed_time(b) for a, b in tev)], dev)
    value = whole_job_mrays(n, world, ms)

    h_v = torch.from_numpy(W["verts"]).pin_memory()
    h_ix = torch.from_numpy(W["prims"].astype(np.int32)).pin_memory()
    h_rays = torch.from_numpy(rays_np.view(np.float32).reshape(-1, 8).copy()).pin_memory()
    h_hits = torch.empty((n, 4), dtype=torch.float32).pin_memory()

    def e2e_step():
        v.copy_(h_v, non_blocking=True)
        ix.copy_(h_ix, non_blocking=True)
        rays.copy_(h_rays, non_blocking=True)
        step()
        h_hits.copy_(hits, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]
    e2e = {"value": round(whole_job_mrays(n, world, e2e_ms), 3), "unit": "Mrays/s",
           "h2d_bytes_per_step": int((h_v.numel() + h_ix.numel() + h_rays.numel()) * 4),
           "d2h_bytes_per_step": int(h_hits.numel() * 4), "ms_per_step": round(e2e_ms, 3)}
    # roofline of the trace kernel: ray (32) + hit, normal, position (40) per
    # ray and the 112-byte solid records and 32-byte nodes it reads
    hbm, src = peaks()
    nn = acc.info()[1]
    alg = n * (32 + 40) + 112 * W["prims"].shape[0] + 32 * nn
    roofline = {"bound": "hbm", "kernel": "solid_trace_kernel<8>",
                "achieved": round(alg / (tms * 1e-3) / 1e9, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(alg / (tms * 1e-3) / 1e9 / hbm, 4), "peak_source": src,
                "traffic": None, "algorithmic_bytes_per_launch": int(alg),
                "note": "unique bytes; the walk is FP64 compute bound (every box on the "
                        "ray's line is visited, as in the reference)"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        got = hits.cpu().numpy()[:: 97]
        want, _, _ = O.OracleSolids(8, W["verts"], W["prims"]).trace(rays_np[:: 97])
        if not np.array_equal(got.view(np.uint32), want.view(np.float32).reshape(-1, 4)
                              .view(np.uint32)):
            raise SystemExit("solid hits differ from the oracle")
        cv, tb, tt, ns, kind = cpu_reference_solids(W)
        cpu = {"value": round(cv, 3), "unit": "Mrays/s", "cores": os.cpu_count(),
               "kind": kind, "sample": f"full Build32 + every ray ({ns}), OpenMP over "
                                       f"{os.cpu_count()} threads",
               "build_s": round(tb, 3), "trace_s": round(tt, 3)}
    line = {"metric": METRIC_SOLIDS, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "trace_ms": round(tms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE["solids"], "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)"),
            "clocks": clk.summary(), "e2e": e2e, "gpu_launches": int(launches),
            "roofline": roofline, "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(line), flush=True)
    acc.close()
    dist_teardown()


def check_line(L, acc, rays, n, hits, nrm):
    from surface_b200._lib import check
    check(L.srt_line_trace(acc.h, rays.data_ptr(), n, hits.data_ptr(), nrm.data_ptr(), None))


# ---------------------------------------------------------------- batched
def run_batched(args, W):
    """One step = every scene built and traced.  Timed twice per step, each
    bracketed by CUDA events on the launching stream with an L2 flush before:
    (a) the batch (srt_batch_build_trace: one launch sequence over all scenes,
    autotuned, replayed from a CUDA graph), (b) the per-scene plain loop
    (srt_accel_build_triangles + srt_trace_closest per scene, one accel per
    scene, same stream).  value = rays / batch step time."""
    import ctypes as C

    import torch

    import surface_b200 as sb
    from surface_b200 import _lib
    from surface_b200.batch import TriangleBatch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    B = W["B"]
    fo, ro = B["face_offsets"], B["ray_offsets"]
    ns = fo.size - 1
    nr = int(ro[-1])
    v = torch.as_tensor(B["vertices"], device=dev)
    f = torch.as_tensor(B["faces"].view(np.int32), device=dev)
    r = torch.as_tensor(B["rays"].view(np.float32).reshape(-1, 8), device=dev)
    hits = torch.empty((nr, 4), dtype=torch.float32, device=dev)
    hits_loop = torch.empty((nr, 4), dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    tb = TriangleBatch(local)

    def batch_step():
        tb.build_trace(v, f, fo, r, ro, hits=hits)

    # the per-scene loop straight through the C ABI (no Python wrapper cost)
    L = _lib.load()
    ctx = sb.Context(local)
    ctx.use_torch_stream()
    accs = []
    for _ in range(ns):
        h = C.c_void_p()
        _lib.check(L.srt_accel_create(ctx.h, _lib.SRT_TRIANGLES, C.byref(h)))
        accs.append(h)
    nv = v.shape[0]
    vp, fp, rp, hp = v.data_ptr(), f.data_ptr(), r.data_ptr(), hits_loop.data_ptr()
    build = L.srt_accel_build_triangles
    trace = L.srt_trace_closest
    chk = _lib.check

    def loop_step():
        for s in range(ns):
            a, b = int(fo[s]), int(fo[s + 1])
            chk(build(accs[s], vp, nv, fp + 12 * a, b - a))
            x, y = int(ro[s]), int(ro[s + 1])
            chk(trace(accs[s], rp + 32 * x, y - x, hp + 16 * x, None))

    for _ in range(max(args.warmup, 3)):
        batch_step()
        loop_step()
    torch.cuda.synchronize()
    _lib.check(L.srt_ctx_synchronize(ctx.h))
    same = torch.equal(hits.view(torch.int32), hits_loop.view(torch.int32))
    block, rpt, captured, kpc = tb.config()
    tuned = tb.tuning()

    # traversal work counters of every scene (one untimed pass) for the roofline
    st = torch.zeros(4, dtype=torch.int64, device=dev)
    opts = _lib.TraceOpts(None, None, None, None, None, st.data_ptr(), 0, 0)
    for s in range(ns):
        x, y = int(ro[s]), int(ro[s + 1])
        _lib.check(trace(accs[s], rp + 32 * x, y - x, hp + 16 * x, C.byref(opts)))
    torch.cuda.synchronize()
    stats = st.cpu().numpy().astype(np.float64)[:3]

    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.keep_busy(batch_step, torch.cuda.synchronize)
        l_b0 = tb.launches()
        l_l0 = L.srt_ctx_launch_count(ctx.h)
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            batch_step()
            ev[k][1].record()
            flush.zero_()
            ev[k][2].record()
            loop_step()
            ev[k][3].record()
        torch.cuda.synchronize()
        launches = tb.launches() - l_b0
        loop_launches = L.srt_ctx_launch_count(ctx.h) - l_l0
        clk.keep_busy(batch_step, torch.cuda.synchronize, extra=1)
    barrier()
    b_ms = [e[0].elapsed_time(e[1]) for e in ev]
    l_ms = [e[2].elapsed_time(e[3]) for e in ev]
    tb_tot, tl_tot = max_over_ranks([sum(b_ms), sum(l_ms)], dev)
    ms_per_step = tb_tot / args.steps
    loop_ms = tl_tot / args.steps
    value = whole_job_mrays(nr, world, ms_per_step)

    # ---- e2e: scenes and rays copied in from pinned host memory, hits out
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_v = pin(B["vertices"])
    h_f = pin(B["faces"].view(np.int32))
    h_r = pin(B["rays"].view(np.float32).reshape(-1, 8))
    h_h = torch.empty((nr, 4), dtype=torch.float32).pin_memory()

    def e2e_step():
        v.copy_(h_v, non_blocking=True)
        f.copy_(h_f, non_blocking=True)
        r.copy_(h_r, non_blocking=True)
        batch_step()
        h_h.copy_(hits, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]
    e2e_value = whole_job_mrays(nr, world, e2e_ms)
    h2d = (h_v.numel() + h_f.numel() + h_r.numel()) * 4
    d2h = h_h.numel() * 4

    # ---- roofline of the whole batched step (build + trace in one graph):
    # traversal bytes from the work counters + build bytes per primitive
    hbm, src = peaks()
    nprim = int(fo[-1])
    trace_bytes = algorithmic_bytes_per_ray("tri", stats, nr) * nr
    build_bytes = nprim * BUILD_BYTES_PER_TRI
    achieved = (trace_bytes + build_bytes) / (ms_per_step * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "whole batched step (graph)",
                "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_source": src, "traffic": None,
                "algorithmic_bytes_per_step": int(trace_bytes + build_bytes),
                "visits_per_ray": [round(float(x) / nr, 3) for x in stats]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cv, ctb, ctt, cns, ck = cpu_reference_batched(W)
        cpu = {"value": round(cv, 4), "unit": "Mrays/s", "cores": os.cpu_count(),
               "kind": ck, "build_s": round(ctb, 3), "trace_s": round(ctt, 3),
               "sample": f"Build32 of all 64 scenes + every ray of each ({cns} of "
                         f"{nr})"}
    for a in accs:
        L.srt_accel_destroy(a)
    if rank == 0:
        line = {
            "metric": METRIC_BATCH, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)",
                           parallelism=f"replicas x{world}"),
            "per_scene_loop_ms": round(loop_ms, 4),
            "speedup_vs_per_scene_loop": round(loop_ms / ms_per_step, 3),
            "batch_launch_shape": {"block": block, "rays_per_grab": rpt,
                                   "graph_captured": captured, "kernels_per_call": kpc},
            "autotuned": tuned,
            "loop_kernels_per_step": int(loop_launches // args.steps),
            "hits_identical_to_loop": bool(same),
            "clocks": clk.summary(),
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    tb.close()
    dist_teardown()


# ---------------------------------------------------------------- particles
def run_particles(args, W):
    """One step = one frame f = k mod 10 of the advected cloud (frames made on
    the device before timing): LBVH rebuild from the frame's centres, 2048^2
    primaries with hit normals, srt_spawn_secondary (one hemisphere ray per
    hit, ray order), secondaries traced with prev_normals (self-hit rule).
    value = (primaries + secondaries) / step time."""
    import ctypes as C

    import torch

    import surface_b200 as sb
    from surface_b200 import _lib
    from surface_b200 import scenes as S

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    nf = W["frames"]
    frames = S.particle_frames(W["verts"], nf, device=dev)
    rad = torch.as_tensor(W["radius"], device=dev)
    npart = int(rad.numel())
    nr = W["rays"].size
    rays = torch.as_tensor(W["rays"].view(np.float32).reshape(-1, 8), device=dev)
    h1 = torch.empty((nr, 4), device=dev)
    n1 = torch.empty((nr, 3), device=dev)
    sec = torch.empty((nr, 8), device=dev)
    sn = torch.empty((nr, 3), device=dev)
    h2 = torch.empty((nr, 4), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    L = _lib.load()
    chk = _lib.check
    ctx = sb.Context(local)
    ctx.use_torch_stream()
    acc = C.c_void_p()
    chk(L.srt_accel_create(ctx.h, _lib.SRT_SPHERES, C.byref(acc)))
    cnt = C.c_uint32()

    def build(k):
        chk(L.srt_accel_build_spheres(acc, frames[k % nf].data_ptr(), rad.data_ptr(),
                                      C.c_float(0.0), npart))

    def primaries(stats=None):
        o = _lib.TraceOpts(None, None, None, None, n1.data_ptr(), stats, 0, 0)
        chk(L.srt_trace_closest(acc, rays.data_ptr(), nr, h1.data_ptr(), C.byref(o)))

    def secondaries(k):
        chk(L.srt_spawn_secondary(ctx.h, rays.data_ptr(), h1.data_ptr(), n1.data_ptr(), nr,
                                  C.c_uint64(k), sec.data_ptr(), sn.data_ptr(), C.byref(cnt)))
        o = _lib.TraceOpts(sn.data_ptr(), None, None, None, None, None, 0, 0)
        chk(L.srt_trace_closest(acc, sec.data_ptr(), cnt.value, h2.data_ptr(), C.byref(o)))
        return cnt.value

    def step(k=0):
        build(k)
        primaries()
        return secondaries(k)

    for k in range(max(args.warmup, 3)):
        step(k)
    torch.cuda.synchronize()
    # primary traversal work counters for the roofline (untimed)
    build(0)
    st = torch.zeros(4, dtype=torch.int64, device=dev)
    primaries(st.data_ptr())
    torch.cuda.synchronize()
    stats_all = st.cpu().numpy().astype(np.float64)
    stats = stats_all[:3]
    sec0 = secondaries(0)

    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    nsec = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.keep_busy(step, torch.cuda.synchronize)
        launches0 = L.srt_ctx_launch_count(ctx.h)
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            build(k)
            ev[k][1].record()
            primaries()
            ev[k][2].record()
            nsec.append(secondaries(k))
            ev[k][3].record()
        torch.cuda.synchronize()
        launches = L.srt_ctx_launch_count(ctx.h) - launches0
        clk.keep_busy(step, torch.cuda.synchronize, extra=1)
    barrier()
    b_ms = [e[0].elapsed_time(e[1]) for e in ev]
    p_ms = [e[1].elapsed_time(e[2]) for e in ev]
    s_ms = [e[2].elapsed_time(e[3]) for e in ev]
    total_ms = max_over_ranks([sum(b_ms) + sum(p_ms) + sum(s_ms)], dev)[0]
    ms_per_step = total_ms / args.steps
    rays_per_step = nr + statistics.mean(nsec)
    value = whole_job_mrays(rays_per_step, world, ms_per_step)

    # ---- e2e: centres, radii and primaries from pinned host memory, both
    # hit arrays back to pinned host memory, every step
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_pos = pin(W["verts"])
    h_rad = pin(W["radius"])
    h_rays = pin(W["rays"].view(np.float32).reshape(-1, 8))
    h_h1 = torch.empty((nr, 4)).pin_memory()
    h_h2 = torch.empty((nr, 4)).pin_memory()

    def e2e_step(k=0):
        chk(L.srt_accel_build_spheres(acc, h_pos.data_ptr(), h_rad.data_ptr(), C.c_float(0.0),
                                      npart))
        o = _lib.TraceOpts(None, None, None, None, n1.data_ptr(), None, 0, 0)
        chk(L.srt_trace_closest(acc, h_rays.data_ptr(), nr, h1.data_ptr(), C.byref(o)))
        c = secondaries(k)
        h_h1.copy_(h1, non_blocking=True)
        h_h2[:c].copy_(h2[:c], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return c

    e2e_warmup(e2e_step, args)
    e2e_s, e2e_c = [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_c.append(e2e_step())
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]
    e2e_value = whole_job_mrays(nr + statistics.mean(e2e_c), world, e2e_ms)
    h2d = (h_pos.numel() + h_rad.numel() + h_rays.numel()) * 4
    d2h = int(16 * (nr + statistics.mean(e2e_c)))

    hbm, src = peaks()
    bpr = algorithmic_bytes_per_ray("sphere", stats, nr)
    pr_ms = statistics.mean(p_ms)
    achieved = bpr * nr / (pr_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "primary trace", "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "peak_source": src, "traffic": None,
                "algorithmic_bytes_per_ray": round(bpr, 1),
                "visits_per_ray": [round(float(x) / nr, 3) for x in stats],
                "reference_walk_rays": int(stats_all[3])}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cv, ctb, ctt, cns, ck = cpu_reference_particles(W)
        cpu = {"value": round(cv, 4), "unit": "Mrays/s", "cores": os.cpu_count(),
               "kind": ck, "build_s": round(ctb, 3), "trace_s": round(ctt, 3),
               "sample": f"Build32 of frame 0 + every primary and the secondaries of "
                         f"its hits ({cns} rays)"}
    L.srt_accel_destroy(acc)
    if rank == 0:
        line = {
            "metric": METRIC_PART, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE["sphere"],
            "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)",
                           parallelism=f"replicas x{world}"),
            "build_ms": round(statistics.mean(b_ms), 4),
            "primary_trace_ms": round(pr_ms, 4),
            "secondary_ms": round(statistics.mean(s_ms), 4),
            "secondary_rays_per_step": round(statistics.mean(nsec), 1),
            "secondary_rays_frame0": int(sec0),
            "clocks": clk.summary(),
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    dist_teardown()


# ---------------------------------------------------------------- frame
def run_frame(args, W):
    """One step = one frame of a resident scene: srt_camera_rays,
    srt_trace_closest, srt_framebuffer_write (RGBA8 + depth).  e2e: the same
    calls with the camera struct as the host input and the colour and depth
    buffers copied back every frame."""
    import ctypes as C

    import torch

    import surface_b200 as sb
    from surface_b200 import _lib
    from surface_b200 import camera as K

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    L = _lib.load()
    chk = _lib.check
    ctx = sb.Context(local)
    ctx.use_torch_stream()
    acc = C.c_void_p()
    chk(L.srt_accel_create(ctx.h, _lib.SRT_TRIANGLES, C.byref(acc)))
    v = torch.as_tensor(W["verts"], device=dev)
    f = torch.as_tensor(W["prims"].view(np.int32), device=dev)
    chk(L.srt_accel_build_triangles(acc, v.data_ptr(), v.shape[0], f.data_ptr(), f.shape[0]))
    cam = K.make_camera(**W["cam"])
    nr = W["cam"]["width"] * W["cam"]["height"]
    rays = torch.empty((nr, 8), device=dev)
    pix = torch.empty((nr,), dtype=torch.int32, device=dev)
    hits = torch.empty((nr, 4), device=dev)
    color = torch.zeros((cam.height, cam.width, 4), dtype=torch.uint8, device=dev)
    depth = torch.zeros((cam.height, cam.width), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    cnt = C.c_uint32()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]

    def step(e=None):
        if e: e[0].record()
        chk(L.srt_camera_rays(ctx.h, C.byref(cam), rays.data_ptr(), pix.data_ptr(),
                              C.byref(cnt)))
        if e: e[1].record()
        chk(L.srt_trace_closest(acc, rays.data_ptr(), cnt.value, hits.data_ptr(), None))
        if e: e[2].record()
        chk(L.srt_framebuffer_write(ctx.h, C.byref(cam), hits.data_ptr(), pix.data_ptr(),
                                    None, cnt.value, 0, color.data_ptr(), depth.data_ptr()))
        if e: e[3].record()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    st = torch.zeros(4, dtype=torch.int64, device=dev)
    opts = _lib.TraceOpts(None, None, None, None, None, st.data_ptr(), 0, 0)
    chk(L.srt_trace_closest(acc, rays.data_ptr(), cnt.value, hits.data_ptr(), C.byref(opts)))
    torch.cuda.synchronize()
    stats = st.cpu().numpy().astype(np.float64)[:3]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.keep_busy(step, torch.cuda.synchronize)
        launches0 = L.srt_ctx_launch_count(ctx.h)
        for k in range(args.steps):
            flush.zero_()
            step(ev[k])
        torch.cuda.synchronize()
        launches = L.srt_ctx_launch_count(ctx.h) - launches0
        clk.keep_busy(step, torch.cuda.synchronize, extra=1)
    barrier()
    r_ms = [e[0].elapsed_time(e[1]) for e in ev]
    t_ms = [e[1].elapsed_time(e[2]) for e in ev]
    w_ms = [e[2].elapsed_time(e[3]) for e in ev]
    total = max_over_ranks([sum(r_ms) + sum(t_ms) + sum(w_ms)], dev)[0]
    ms_per_step = total / args.steps
    value = whole_job_mrays(nr, world, ms_per_step)

    # ---- e2e: camera in, colour and depth out, every frame
    h_color = torch.empty_like(color, device="cpu").pin_memory()
    h_depth = torch.empty_like(depth, device="cpu").pin_memory()

    def e2e_step():
        step()
        h_color.copy_(color, non_blocking=True)
        h_depth.copy_(depth, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]

    hbm, src = peaks()
    bpr = algorithmic_bytes_per_ray("tri", stats, nr)
    tr_ms = statistics.mean(t_ms)
    achieved = bpr * nr / (tr_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "trace", "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "peak_source": src, "traffic": None,
                "algorithmic_bytes_per_ray": round(bpr, 1),
                "visits_per_ray": [round(float(x) / nr, 3) for x in stats]}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        vals = [cpu_reference_frame(W) for _ in range(3)]
        cv, ctr, ctt, cns, ck = sorted(vals)[1]
        cpu = {"value": round(cv, 4), "unit": "Mrays/s", "cores": os.cpu_count(), "kind": ck,
               "rays_write_s": round(ctr, 4), "trace_s": round(ctt, 4),
               "sample": f"every pixel ({cns} rays), median of 3: eye rays and write of "
                         f"the CPU restatement, Traverse of the reference"}
    L.srt_accel_destroy(acc)
    if rank == 0:
        line = {
            "metric": METRIC_FRAME, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)",
                           parallelism=f"replicas x{world}"),
            "camera_rays_ms": round(statistics.mean(r_ms), 4),
            "trace_ms": round(tr_ms, 4),
            "framebuffer_write_ms": round(statistics.mean(w_ms), 4),
            "clocks": clk.summary(),
            "e2e": {"value": round(whole_job_mrays(nr, world, e2e_ms), 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": C.sizeof(cam),
                    "d2h_bytes_per_step": int(h_color.numel() + 4 * h_depth.numel()),
                    "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    dist_teardown()


def run_scene(args, W):
    """One step = one frame of a resident multi-element scene, as glFinish
    runs it: srt_scene_build (RenderGraph::Build), srt_camera_rays,
    srt_scene_trace, srt_framebuffer_write (RGBA8 + depth).  e2e: the same
    calls with the camera struct as the host input and the colour and depth
    buffers copied back every frame."""
    import ctypes as C

    import torch

    import surface_b200 as sb
    from surface_b200 import _lib
    from surface_b200 import camera as K

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)
    L = _lib.load()
    chk = _lib.check
    ctx = sb.Context(local)
    ctx.use_torch_stream()
    E = W["E"]
    accs, keep = [], []
    for a in E["accels"]:
        h = C.c_void_p()
        kind = {0: _lib.SRT_TRIANGLES, 1: _lib.SRT_TETRAHEDRA, 2: _lib.SRT_SPHERES}[a["kind"]]
        chk(L.srt_accel_create(ctx.h, kind, C.byref(h)))
        v = torch.as_tensor(a["verts"], device=dev)
        if a["kind"] == 2:
            r = torch.as_tensor(a["radius"], device=dev)
            chk(L.srt_accel_build_spheres(h, v.data_ptr(), r.data_ptr(), C.c_float(0.0),
                                          v.shape[0]))
            keep += [v, r]
        else:
            f = torch.as_tensor(a["faces"].view(np.int32), device=dev)
            build = (L.srt_accel_build_triangles if a["kind"] == 0
                     else L.srt_accel_build_tetrahedra)
            chk(build(h, v.data_ptr(), v.shape[0], f.data_ptr(), f.shape[0]))
            keep += [v, f]
        accs.append(h)
    sc = C.c_void_p()
    chk(L.srt_scene_create(ctx.h, C.byref(sc)))
    for el in E["elements"]:
        T = np.ascontiguousarray(el["T"], np.float64).reshape(16)
        chk(L.srt_scene_add_element(sc, accs[el["accel"]], T.ctypes.data, None))
    cam = K.make_camera(**W["cam"])
    nr = W["cam"]["width"] * W["cam"]["height"]
    rays = torch.empty((nr, 8), device=dev)
    pix = torch.empty((nr,), dtype=torch.int32, device=dev)
    hits = torch.empty((nr, 4), device=dev)
    elem = torch.empty((nr,), dtype=torch.int32, device=dev)
    color = torch.zeros((cam.height, cam.width, 4), dtype=torch.uint8, device=dev)
    depth = torch.zeros((cam.height, cam.width), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    cnt = C.c_uint32()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(args.steps)]

    def step(e=None, stats=None):
        if e: e[0].record()
        chk(L.srt_scene_build(sc))
        if e: e[1].record()
        chk(L.srt_camera_rays(ctx.h, C.byref(cam), rays.data_ptr(), pix.data_ptr(),
                              C.byref(cnt)))
        if e: e[2].record()
        chk(L.srt_scene_trace(sc, rays.data_ptr(), cnt.value, None, None, hits.data_ptr(),
                              elem.data_ptr(), stats))
        if e: e[3].record()
        chk(L.srt_framebuffer_write(ctx.h, C.byref(cam), hits.data_ptr(), pix.data_ptr(),
                                    None, cnt.value, 0, color.data_ptr(), depth.data_ptr()))
        if e: e[4].record()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    chk(L.srt_ctx_synchronize(ctx.h))  # surfaces any kernel limit flag
    st = torch.zeros(5, dtype=torch.int64, device=dev)
    step(None, st.data_ptr())
    torch.cuda.synchronize()
    stats = st.cpu().numpy().astype(np.float64)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.keep_busy(step, torch.cuda.synchronize)
        launches0 = L.srt_ctx_launch_count(ctx.h)
        for k in range(args.steps):
            flush.zero_()
            step(ev[k])
        torch.cuda.synchronize()
        launches = L.srt_ctx_launch_count(ctx.h) - launches0
        clk.keep_busy(step, torch.cuda.synchronize, extra=1)
    barrier()
    chk(L.srt_ctx_synchronize(ctx.h))
    parts = [[e[j].elapsed_time(e[j + 1]) for e in ev] for j in range(4)]
    total = max_over_ranks([sum(sum(p) for p in parts)], dev)[0]
    ms_per_step = total / args.steps
    value = whole_job_mrays(nr, world, ms_per_step)

    h_color = torch.empty_like(color, device="cpu").pin_memory()
    h_depth = torch.empty_like(depth, device="cpu").pin_memory()

    def e2e_step():
        step()
        h_color.copy_(color, non_blocking=True)
        h_depth.copy_(depth, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]

    hbm, src = peaks()
    ntop, nwalk, br, lf, pr = (float(x) / nr for x in stats)
    # ray (32) + hit (16) + element (4) + top-level nodes (72) + per element
    # walk its record (424) + branch nodes (64) + primitive records (48: the
    # triangle size; tets 52, spheres 20)
    bpr = 32 + 16 + 4 + 72 * ntop + 424 * nwalk + 64 * br + 48 * pr
    tr_ms = statistics.mean(parts[2])
    achieved = bpr * nr / (tr_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "srt_scene_trace (top, walk and resolve kernels)",
                "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "peak_source": src, "traffic": None,
                "algorithmic_bytes_per_ray": round(bpr, 1),
                "visits_per_ray": {"top_nodes": round(ntop, 3), "element_walks": round(nwalk, 3),
                                   "branch": round(br, 3), "leaf": round(lf, 3),
                                   "prims": round(pr, 3)}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        vals = [cpu_reference_scene(W) for _ in range(3)]
        cv, ctr, ctt, cns, ck = sorted(vals)[1]
        cpu = {"value": round(cv, 4), "unit": "Mrays/s", "cores": os.cpu_count(), "kind": ck,
               "build_rays_write_s": round(ctr, 4), "trace_s": round(ctt, 4),
               "sample": f"top-level build, eye rays, scene trace and write of every "
                         f"pixel ({cns} rays, OpenMP); median of 3, CPU restatement"}
    L.srt_scene_destroy(sc)
    for h in accs:
        L.srt_accel_destroy(h)
    if rank == 0:
        line = {
            "metric": METRIC_SCENE, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE["scene"],
            "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)",
                           parallelism=f"replicas x{world}"),
            "top_build_ms": round(statistics.mean(parts[0]), 4),
            "camera_rays_ms": round(statistics.mean(parts[1]), 4),
            "trace_ms": round(tr_ms, 4),
            "framebuffer_write_ms": round(statistics.mean(parts[3]), 4),
            "clocks": clk.summary(),
            "e2e": {"value": round(whole_job_mrays(nr, world, e2e_ms), 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": C.sizeof(cam),
                    "d2h_bytes_per_step": int(h_color.numel() + 4 * h_depth.numel()),
                    "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    dist_teardown()


# ---------------------------------------------------------------- GPU arm
def run_ours(args, W):
    import torch

    import surface_b200 as sb
    from surface_b200 import _lib

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # all work (ours and the timing events) on one dedicated stream
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    world, rank = dist_setup(dev)

    kind = W["kind"]
    ctx = sb.Context(local)
    Acc = {"tet": sb.TetraAccel, "tri": sb.TriangleAccel, "sphere": sb.ParticleAccel}[kind]
    acc = Acc(ctx)
    nr = W["rays"].size
    verts = torch.as_tensor(W["verts"], device=dev)
    prims = torch.as_tensor(W["prims"].astype(np.int32), device=dev) if "prims" in W else None
    radius = torch.as_tensor(W["radius"], device=dev) if "radius" in W else None
    scalar = torch.as_tensor(W["scalar"], device=dev) if "scalar" in W else None
    rays = torch.as_tensor(W["rays"].view(np.float32).reshape(-1, 8), device=dev)
    hits = torch.empty((nr, 4), dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def build():
        if kind == "tri":
            acc.Build32(sb.Mesh(verts, prims))
        elif kind == "tet":
            acc.Build32(sb.Tetrahedron(verts, prims))
        else:
            acc.Build32(sb.Particles(verts, radius))

    def trace():
        if kind == "tet":
            return acc.Traverse(rays, hits=hits, vertex_scalar=scalar, want_scalar=True)
        return acc.Traverse(rays, hits=hits)

    def step():
        build()
        trace()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    # traversal work counters for the roofline (one extra untimed pass)
    st = torch.zeros(4, dtype=torch.int64, device=dev)
    L = _lib.load()
    opts = _lib.TraceOpts(None, None, scalar.data_ptr() if scalar is not None else None,
                          None, None, st.data_ptr(), 0, 0)
    ctx.use_torch_stream()
    _lib.check(L.srt_trace_closest(acc.h, rays.data_ptr(), nr, hits.data_ptr(),
                                   __import__("ctypes").byref(opts)))
    torch.cuda.synchronize()
    stats_all = st.cpu().numpy().astype(np.float64)
    stats = stats_all[:3]

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.keep_busy(step, torch.cuda.synchronize)
        launches0 = L.srt_ctx_launch_count(ctx.h)
        for k in range(args.steps):
            flush.zero_()
            e0, e1, e2 = ev[k]
            e0.record()
            build()
            e1.record()
            trace()
            e2.record()
        torch.cuda.synchronize()
        launches = L.srt_ctx_launch_count(ctx.h) - launches0
        clk.keep_busy(step, torch.cuda.synchronize, extra=1)
    barrier()
    build_ms = [e[0].elapsed_time(e[1]) for e in ev]
    trace_ms = [e[1].elapsed_time(e[2]) for e in ev]
    total_ms = max_over_ranks([sum(b + t for b, t in zip(build_ms, trace_ms))], dev)[0]
    ms_per_step = total_ms / args.steps
    value = whole_job_mrays(nr, world, ms_per_step)

    # ---- e2e through the C ABI with pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_verts = pin(W["verts"])
    h_prims = pin(W["prims"]) if "prims" in W else None
    h_rad = pin(W["radius"]) if "radius" in W else None
    h_rays = pin(W["rays"].view(np.float32).reshape(-1, 8))
    h_hits = torch.empty((nr, 4), dtype=torch.float32).pin_memory()
    h_scal = torch.empty((nr,), dtype=torch.float32).pin_memory()
    import ctypes as C
    e2e_acc = C.c_void_p()
    _lib.check(L.srt_accel_create(ctx.h, acc.KIND, C.byref(e2e_acc)))
    ctx.use_own_stream()
    d_scalar = scalar

    def e2e_step():
        if kind == "tri":
            _lib.check(L.srt_accel_build_triangles(e2e_acc, h_verts.data_ptr(),
                                                   h_verts.shape[0], h_prims.data_ptr(),
                                                   h_prims.shape[0]))
        elif kind == "tet":
            _lib.check(L.srt_accel_build_tetrahedra(e2e_acc, h_verts.data_ptr(),
                                                    h_verts.shape[0], h_prims.data_ptr(),
                                                    h_prims.shape[0]))
        else:
            _lib.check(L.srt_accel_build_spheres(e2e_acc, h_verts.data_ptr(),
                                                 h_rad.data_ptr(), C.c_float(0.0),
                                                 h_verts.shape[0]))
        o = _lib.TraceOpts(None, None, d_scalar.data_ptr() if d_scalar is not None else None,
                           h_scal.data_ptr() if kind == "tet" else None, None, None, 0, 0)
        _lib.check(L.srt_trace_closest(e2e_acc, h_rays.data_ptr(), nr, h_hits.data_ptr(),
                                       C.byref(o)))

    e2e_warmup(e2e_step, args)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    L.srt_accel_destroy(e2e_acc)
    e2e_ms = max_over_ranks([1e3 * sum(e2e_s) / len(e2e_s)], dev)[0]
    e2e_value = whole_job_mrays(nr, world, e2e_ms)
    h2d = (h_verts.numel() * 4 + (h_prims.numel() * 4 if h_prims is not None else 0)
           + (h_rad.numel() * 4 if h_rad is not None else 0) + h_rays.numel() * 4)
    d2h = h_hits.numel() * 4 + (h_scal.numel() * 4 if kind == "tet" else 0)

    # ---- roofline of the dominant kernel (traversal)
    hbm, src = peaks()
    bpr = algorithmic_bytes_per_ray(kind, stats, nr)
    tr_ms = statistics.mean(trace_ms)
    achieved = bpr * nr / (tr_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "trace", "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "peak_source": src, "traffic": profiled_traffic(kind),
                "traffic_source": (f"profiles/{TRAFFIC_PROFILE[kind]} (first-pass kernel)"
                                   if kind in TRAFFIC_PROFILE else None),
                "algorithmic_bytes_per_ray": round(bpr, 1),
                "visits_per_ray": [round(float(x) / nr, 3) for x in stats],
                "reference_walk_rays": int(stats_all[3])}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, tb, tt, ns, ck = cpu_reference_step(W)
        cpu = {"value": round(v, 4), "unit": "Mrays/s", "cores": os.cpu_count(),
               "kind": ck, "build_s": round(tb, 4), "trace_s": round(tt, 4),
               "sample": f"the full step: Build32 + every ray ({ns} of {nr}), OpenMP "
                         f"over {os.cpu_count()} threads"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[kind], "data": "synthetic",
            "config": dict(W["config"], l2="flushed between steps (256 MiB write)",
                           parallelism=f"replicas x{world}"),
            "build_ms": round(statistics.mean(build_ms), 4),
            "trace_ms": round(tr_ms, 4),
            "trace_mrays": round(nr / (tr_ms * 1e-3) / 1e6, 2),
            "clocks": clk.summary(),
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    dist_teardown()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tri",
                    choices=["tet", "tri", "particles", "volume", "batched", "frame",
                             "scene", "texture", "lines", "solids", "volume_nu"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.impl == "reference" and int(os.environ.get("RANK", "0")) != 0:
        return  # the CPU reference runs on rank 0 alone; other ranks exit 0
    if args.impl == "reference" and args.workload in ("volume", "volume_nu"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference's march is GLSL shader code that needs its closed "
                          "prebuilt compiler; no reference CPU march exists"}), flush=True)
        return
    W = make_workload(args.workload)
    if args.workload in ("volume", "volume_nu"):
        run_volume(args, W)
        return
    if args.impl == "reference":
        run_reference_arm(args, W)
    elif args.workload == "batched":
        run_batched(args, W)
    elif args.workload == "particles":
        run_particles(args, W)
    elif args.workload == "frame":
        run_frame(args, W)
    elif args.workload == "scene":
        run_scene(args, W)
    elif args.workload == "texture":
        run_texture(args, W)
    elif args.workload == "lines":
        run_lines(args, W)
    elif args.workload == "solids":
        run_solids(args, W)
    else:
        run_ours(args, W)


if __name__ == "__main__":
    main()
