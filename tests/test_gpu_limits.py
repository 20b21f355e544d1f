"""The traversal's device-side limit path: a walk that reaches its step cap
stops, the kernel records the event in the context's error word, the call
(or srt_ctx_synchronize) reports SRT_ERR_LIMIT, and the context traces
correctly afterwards.  The cap is lowered per call through
srt_trace_opts.max_iter, so a normal scene reaches it; the kernels return at
the cap, nothing waits or faults.  The reference asserts on its stack depth
instead (render/render_accel_triangle.cc:2661)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import surface_b200 as sb  # noqa: E402
from oracle import oracle as O  # noqa: E402
from surface_b200 import _lib  # noqa: E402
from surface_b200 import scenes as S  # noqa: E402

from conftest import bits  # noqa: E402

pytestmark = pytest.mark.gpu


def _scene(kind):
    if kind == O.TRI:
        v, f = S.displaced_octasphere(6, seed=2)
        acc = sb.TriangleAccel()
        acc.Build32(sb.Mesh(v, f))
        return acc, O.OracleAccel(O.TRI, v, f), S.pinhole_rays(128, 128, (0, 0, 3), (0, 0, 0))
    if kind == O.TET:
        v, f, _ = S.tet_grid(16, seed=2)
        acc = sb.TetraAccel()
        acc.Build32(sb.Tetrahedron(v, f))
        return acc, O.OracleAccel(O.TET, v, f), S.ortho_rays(128, 128)
    p, r = S.particles(50_000, seed=2)
    acc = sb.ParticleAccel()
    acc.Build32(sb.Particles(p, r))
    return acc, O.OracleAccel(O.SPHERE, p, None, r), S.pinhole_rays(
        128, 128, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)


@pytest.mark.parametrize("kind", [O.TRI, O.TET, O.SPHERE])
@pytest.mark.parametrize("single", [False, True])
def test_step_cap_reports_limit_and_context_recovers(kind, single):
    acc, o, rays = _scene(kind)
    # host arrays: the call synchronises and reports the kernels' limit hit
    with pytest.raises(sb.SurfaceError) as ei:
        acc.Traverse(rays, max_iter=4, single_pass=single)
    assert ei.value.status == _lib.SRT_ERR_LIMIT
    # device arrays: asynchronous; srt_ctx_synchronize reports it
    rt = torch.as_tensor(rays.view(np.float32).reshape(-1, 8), device="cuda")
    acc.Traverse(rt, max_iter=4, single_pass=single)
    L = _lib.load()
    acc.ctx.use_torch_stream()
    assert L.srt_ctx_synchronize(acc.ctx.h) == _lib.SRT_ERR_LIMIT
    assert L.srt_ctx_synchronize(acc.ctx.h) == _lib.SRT_OK  # reported once
    # the same context then traces exactly
    h = acc.Traverse(rays, single_pass=single)
    want = o.trace(rays)
    for f in ("t", "prim") + (("u", "v") if kind != O.SPHERE else ()):
        assert np.array_equal(bits(h[f]), bits(want[f])), f
    # a cap above what any walk needs changes nothing
    h2 = acc.Traverse(rays, max_iter=1_000_000, single_pass=single)
    assert np.array_equal(h2.view(np.uint32), h.view(np.uint32))
