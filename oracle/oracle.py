"""ctypes bindings to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries live here:

* ``liboracle.so`` -- the plain-C restatement of SURFACE's LBVH build, closest-hit
  traversal, trilinear fetch and volume march (``surface_oracle.c``), built from
  this directory by ``make -C oracle oracle``.
* ``_ref/libsurface_ref.so`` -- the reference's own ``render/`` sources linked
  with ``ref_harness.cc`` (``make -C oracle ref``; needs the reference tree at
  build time, the built library travels with the working tree).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsurface_ref.so")

TRI, TET, SPHERE = 0, 1, 2
MISS = 0xFFFFFFFF

# ray / hit records shared by the oracle, the reference harness and the C ABI
RAY_DTYPE = np.dtype([("org", "<f4", 3), ("prev_prim", "<u4"), ("dir", "<f4", 3),
                      ("prev_t", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("prim", "<u4")])
# shading record of a hit (BuildIntersection's fields; srt_isect in the C ABI)
ISECT_DTYPE = np.dtype([("position", "<f4", 3), ("f0", "<u4"), ("normal", "<f4", 3),
                        ("f1", "<u4"), ("tangent", "<f4", 3), ("f2", "<u4"),
                        ("binormal", "<f4", 3), ("f3", "<u4"), ("d", "<f4", 4)])
# generic node (own box, leaf flag, axis, d0, d1): so_node in surface_oracle.c
NODE_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("leaf", "<i4"),
                       ("axis", "<i4"), ("d0", "<u4"), ("d1", "<u4")])

# test/cctest/test-prefix-tree.cc:10-23 fixture RNG parameters
TMT_MAT1, TMT_MAT2, TMT_TMAT = 0xFA051F40, 0xFFD0FFF4, 0x58D02FFEFFBFFFBC

_P = C.c_void_p
_SZ = C.c_size_t


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _build(target):
    subprocess.run(["make", "-s", "-C", HERE, target], check=True,
                   stdout=subprocess.DEVNULL)


_ORACLE = None
_REF = None


def lib():
    """The restatement library (built on first use if missing)."""
    global _ORACLE
    if _ORACLE is None:
        if not os.path.exists(ORACLE_SO):
            _build("oracle")
        L = C.CDLL(ORACLE_SO)
        L.so_build.restype = _P
        L.so_build.argtypes = [C.c_int, _P, _P, _P, C.c_float, _SZ]
        L.so_build_tet_d.restype = _P
        L.so_build_tet_d.argtypes = [_P, _SZ, _P, _SZ]
        L.so_free.argtypes = [_P]
        L.so_num_nodes.restype = _SZ
        L.so_num_nodes.argtypes = [_P]
        L.so_export.argtypes = [_P, _P, _P, _P, _P, _P]
        L.so_export_karras.argtypes = [_P, _P, _P, _P]
        L.so_canonicalize.restype = C.c_long
        L.so_canonicalize.argtypes = [_P, _SZ, _SZ, _P, _SZ]
        L.so_trace.argtypes = [_P, _P, _SZ, _P, _P, _P, _P, _P, _P, C.c_int]
        L.so_trace2.argtypes = [_P, _P, _SZ, _P, _P, _P, _P, C.c_int]
        L.so_isect_records.argtypes = [_P, _P, _SZ, _P, _P, _P, C.c_int]
        L.so_morton_bits.restype = C.c_uint32
        L.so_morton_bits.argtypes = [C.c_uint32] * 3
        for n in ("so_morton_tris", "so_morton_tets"):
            getattr(L, n).argtypes = [_P, _P, _SZ, _P, _P, _P]
        L.so_morton_points.argtypes = [_P, _SZ, _P, _P, _P]
        L.so_bbox_tris.argtypes = [_P, _P, _SZ, _P, _P]
        L.so_bbox_tets.argtypes = [_P, _P, _SZ, _P, _P]
        L.so_bbox_spheres.argtypes = [_P, _P, C.c_float, _SZ, _P, _P]
        L.so_sort_pairs.argtypes = [_P, _P, _SZ]
        L.so_karras.argtypes = [_P, _SZ, _P, _P, _P]
        L.so_tinymt64_doubles.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32,
                                          C.c_uint64, _SZ, _P]
        L.so_tex3d.argtypes = [_P, _P, _P, _SZ, C.c_int, C.c_int, C.c_int, _P]
        L.so_volume_camera.argtypes = [C.c_int, C.c_int, _P, _P, _P, C.c_float,
                                       _P, _P, _P]
        L.so_volume_fwd_f32.argtypes = [_P, _P, _P, _P, _P, C.c_int]
        L.so_volume_f64.restype = C.c_double
        L.so_volume_f64.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P]
        L.so_volume_fwd_f32_ex.argtypes = [_P, _P, _P, _P, _P, _P, C.c_int]
        L.so_volume_f64_ex.restype = C.c_double
        L.so_volume_f64_ex.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.so_volume_f64_pixels.restype = C.c_double
        L.so_volume_f64_pixels.argtypes = [_P, _P, _P, _P, _P, _P, _SZ]
        L.so_camera_frame.argtypes = [_P, _P, _P, C.c_float, C.c_int, C.c_int, C.c_int, _P]
        L.so_camera_rays.restype = _SZ
        L.so_camera_rays.argtypes = [_P, _P, _P, _P]
        L.so_framebuffer_write.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, _P, _SZ,
                                           C.c_int, _P, _P]
        L.so_stereo_env_ray.argtypes = [_P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_float,
                                        C.c_int, C.c_int, _P, _P]
        L.so_camera_rays_ex.restype = _SZ
        L.so_camera_rays_ex.argtypes = [_P, _P, _P, _P, C.c_uint64, C.c_uint64, _P, _P]
        L.so_framebuffer_write_ex.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P,
                                              _SZ, C.c_int, _P, _P]
        L.so_tex_fetch.argtypes = [C.c_int, _P, _P, C.c_int, _P, _P, _P, _P, _SZ, _P]
        L.so_sparse_tree.restype = _P
        L.so_sparse_tree.argtypes = [_P, _SZ]
        L.so_sparse_fetch.argtypes = [_P, _P, _P, C.c_int, C.c_int, _P, _P, _SZ, _P]
        L.so_matrix_inverse.argtypes = [_P]
        L.so_element_update.argtypes = [_P, _P, _P, _P, _P, _P, _P]
        L.so_scene_build.restype = _P
        L.so_scene_build.argtypes = [_P, _P, _P, _P, _P, _P, _SZ]
        L.so_scene_free.argtypes = [_P]
        L.so_scene_set_kind.restype = None
        L.so_scene_set_kind.argtypes = [_P, _SZ, C.c_int]
        L.so_scene_top_nodes.restype = _SZ
        L.so_scene_top_nodes.argtypes = [_P, _P, _P, _SZ]
        L.so_scene_candidates.restype = _SZ
        L.so_scene_candidates.argtypes = [_P, _P, _P, _P, _P, _SZ]
        L.so_scene_trace.argtypes = [_P, _P, _SZ, _P, _P, _P, _P, _P, C.c_int, C.c_int]
        L.so_line_build.restype = _P
        L.so_line_build.argtypes = [_P, _P, C.c_float, _P, _SZ, C.c_int, C.c_int, C.c_int]
        L.so_line_free.argtypes = [_P]
        L.so_line_num_nodes.restype = _SZ
        L.so_line_num_nodes.argtypes = [_P]
        L.so_line_depth.restype = C.c_int
        L.so_line_depth.argtypes = [_P]
        L.so_line_export.argtypes = [_P, _P, _P]
        L.so_line_trace.argtypes = [_P, _P, _SZ, _P, _P, C.c_int]
        L.so_solid_build.restype = _P
        L.so_solid_build.argtypes = [C.c_int, _P, _P, _SZ]
        L.so_solid_build_d.restype = _P
        L.so_solid_build_d.argtypes = [C.c_int, _P, _P, _SZ]
        L.so_solid_build_sah.restype = _P
        L.so_solid_build_sah.argtypes = [C.c_int, _P, _P, _P, _SZ]
        L.so_solid_free.argtypes = [_P]
        L.so_solid_num_nodes.restype = _SZ
        L.so_solid_num_nodes.argtypes = [_P]
        L.so_solid_export.argtypes = [_P, _P, _P]
        L.so_solid_trace.argtypes = [_P, _P, _SZ, _P, _P, _P, C.c_int]
        _ORACLE = L
    return _ORACLE


def have_ref():
    return os.path.exists(REF_SO)


def ref():
    """The reference's own code (None when it was never built here)."""
    global _REF
    if _REF is None:
        if not os.path.exists(REF_SO):
            try:
                _build("ref")
            except Exception:
                pass
        if not os.path.exists(REF_SO):
            return None
        L = C.CDLL(REF_SO)
        for k in ("tri", "tet", "sphere"):
            getattr(L, f"ref_{k}_free").argtypes = [_P]
            getattr(L, f"ref_{k}_dump").argtypes = [_P, C.c_char_p]
            getattr(L, f"ref_{k}_bbox").argtypes = [_P, _P, _P]
        L.ref_tri_build.restype = _P
        L.ref_tri_build.argtypes = [_P, _SZ, _P, _SZ]
        L.ref_tet_build.restype = _P
        L.ref_tet_build.argtypes = [_P, _P, _SZ]
        L.ref_tet_build_d.restype = _P
        L.ref_tet_build_d.argtypes = [_P, _P, _SZ]
        L.ref_sphere_build.restype = _P
        L.ref_sphere_build.argtypes = [_P, _P, C.c_float, _SZ]
        L.ref_tri_trace.argtypes = [_P, _P, _SZ, _P, C.c_int, C.c_int]
        L.ref_tet_trace.argtypes = [_P, _P, _SZ, _P, _P, C.c_int, C.c_int]
        L.ref_sphere_trace.argtypes = [_P, _P, _SZ, _P, _P, C.c_int, C.c_int]
        L.ref_tri_trace_isect.argtypes = [_P, _P, _SZ, _P, _P, C.c_int]
        L.ref_tet_trace_isect.argtypes = [_P, _P, _SZ, _P, _P, _P, C.c_int]
        L.ref_sphere_trace_isect.argtypes = [_P, _P, _SZ, _P, _P, _P, C.c_int]
        L.ref_node_sizes.argtypes = [_P]
        L.ref_morton_points.argtypes = [_P, _SZ, _P, _P, _P, C.c_int]
        L.ref_morton_tris.argtypes = [_P, _P, _SZ, _P, _P, _P]
        L.ref_morton_tets.argtypes = [_P, _P, _SZ, _P, _P, _P]
        L.ref_morton_code.restype = C.c_uint32
        L.ref_morton_code.argtypes = [_P, _P, C.c_float]
        L.ref_radix_sort.argtypes = [_P, _P, _SZ]
        L.ref_karras.argtypes = [_P, _SZ, _P, _P, _P]
        L.ref_tex3d.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_int, _P, _SZ,
                                C.c_int, C.c_int, C.c_int, _P]
        L.ref_tinymt64_doubles.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32,
                                           C.c_uint64, _SZ, _P]
        L.ref_camera_frame.argtypes = [_P, _P, _P, C.c_float, C.c_int, C.c_int, C.c_int,
                                       _P]
        L.ref_stereo_env_ray.argtypes = [_P, _P, _P, C.c_float, C.c_float, C.c_float,
                                         C.c_float, C.c_int, C.c_int, _P]
        L.ref_tex_fetch.argtypes = [C.c_int, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P,
                                    _P, C.c_int, _P, C.c_int, _P, C.c_int, _P, _SZ, _P]
        L.ref_sparse_fetch.argtypes = [_P, _SZ, _P, C.c_int, C.c_int, _P, _P, _SZ, _P]
        L.ref_matrix_inverse.argtypes = [_P]
        L.ref_bvh_build.restype = _P
        L.ref_bvh_build.argtypes = [_P, _P, _P, _SZ]
        L.ref_bvh_free.argtypes = [_P]
        L.ref_bvh_nodes.restype = _SZ
        L.ref_bvh_nodes.argtypes = [_P, _P, _P, _SZ]
        L.ref_bvh_trace.restype = _SZ
        L.ref_bvh_trace.argtypes = [_P, _P, _P, _P, _P, _SZ]
        L.ref_line_build.restype = _P
        L.ref_line_build.argtypes = [_P, _P, C.c_float, _P, _SZ, C.c_int, C.c_int, C.c_int]
        L.ref_line_free.argtypes = [_P]
        L.ref_line_dump.argtypes = [_P, C.c_char_p]
        L.ref_line_bbox.argtypes = [_P, _P, _P]
        L.ref_line_trace.argtypes = [_P, _P, _SZ, _P, _P, C.c_int, C.c_int]
        L.ref_solid_build.restype = _P
        L.ref_solid_build.argtypes = [C.c_int, _P, _P, _SZ]
        L.ref_solid_build_d.restype = _P
        L.ref_solid_build_d.argtypes = [C.c_int, _P, _P, _SZ]
        L.ref_solid_build_sah.restype = _P
        L.ref_solid_build_sah.argtypes = [C.c_int, _P, _P, _P, _SZ]
        L.ref_solid_free.argtypes = [_P]
        L.ref_solid_dump.argtypes = [_P, C.c_char_p]
        L.ref_solid_bbox.argtypes = [_P, _P, _P]
        L.ref_solid_trace.argtypes = [_P, _P, _SZ, _P, _P, _P, C.c_int, C.c_int]
        _REF = L
    return _REF


# --------------------------------------------------------------------------
# oracle accel
# --------------------------------------------------------------------------
class OracleAccel:
    """LBVH built by the C restatement; nodes in the reference's sequential
    emission order (depth-first, left first)."""

    def __init__(self, kind, verts, faces=None, radius=None, const_radius=0.0):
        """Tetrahedra with float64 vertices keep double precision
        (isDoublePrecisionPos)."""
        self.kind = kind
        dbl = kind == TET and np.asarray(verts).dtype == np.float64
        self.verts = np.ascontiguousarray(verts, np.float64 if dbl else np.float32).reshape(-1)
        self.faces = None if faces is None else np.ascontiguousarray(faces, np.uint32).reshape(-1)
        self.radius = None if radius is None else np.ascontiguousarray(radius, np.float32)
        n = {TRI: None, TET: None, SPHERE: None}[kind]
        if kind == TRI:
            n = self.faces.size // 3
        elif kind == TET:
            n = self.faces.size // 4
        else:
            n = self.verts.size // 3
        self.n = n
        if dbl:
            self.h = lib().so_build_tet_d(_ptr(self.verts), self.verts.size // 3,
                                          _ptr(self.faces), n)
        else:
            self.h = lib().so_build(kind, _ptr(self.verts), _ptr(self.faces),
                                    _ptr(self.radius), C.c_float(const_radius), n)
        if not self.h:
            raise ValueError("oracle build needs at least 2 primitives")
        nn = lib().so_num_nodes(self.h)
        self.nodes = np.zeros(nn, NODE_DTYPE)
        self.indices = np.zeros(n, np.uint32)
        self.codes = np.zeros(n, np.uint32)
        scene = np.zeros(6, np.float32)
        eps = C.c_double()
        lib().so_export(self.h, _ptr(self.nodes), _ptr(self.indices), _ptr(self.codes),
                        _ptr(scene), C.byref(eps))
        self.scene_bmin, self.scene_bmax = scene[:3].copy(), scene[3:].copy()
        self.eps_scale = eps.value

    def bbox64(self):
        """XxxAccel::BoundingBox: the root node's box, as doubles."""
        return (self.nodes["bmin"][0].astype(np.float64),
                self.nodes["bmax"][0].astype(np.float64))

    def karras(self):
        m = self.n - 1
        child = np.zeros(m, np.uint32)
        lt = np.zeros(m, np.uint8)
        rt = np.zeros(m, np.uint8)
        lib().so_export_karras(self.h, _ptr(child), _ptr(lt), _ptr(rt))
        return child, lt, rt

    def canonical(self):
        return canonicalize(self.nodes, 0)

    def trace(self, rays, prev_normals=None, want_subface=False, want_stats=False,
              nthreads=0, vertex_scalar=None):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        sub = np.zeros(rays.size, np.uint32) if want_subface else None
        st = np.zeros(3, np.uint64)
        pn = None if prev_normals is None else np.ascontiguousarray(prev_normals, np.float32)
        vs = None if vertex_scalar is None else np.ascontiguousarray(vertex_scalar, np.float32)
        so = np.zeros(rays.size, np.float32) if vs is not None else None
        lib().so_trace(self.h, _ptr(rays), rays.size, _ptr(pn), _ptr(hits), _ptr(sub),
                       _ptr(vs), _ptr(so), _ptr(st), nthreads)
        out = [hits]
        if want_subface:
            out.append(sub)
        if vs is not None:
            out.append(so)
        if want_stats:
            out.append(st)
        return out[0] if len(out) == 1 else tuple(out)

    def trace2(self, rays, prev_normals=None, want_subface=False, want_stats=False,
               nthreads=0):
        """The product's two-pass walk, restated (for checking it on the CPU)."""
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        sub = np.zeros(rays.size, np.uint32) if want_subface else None
        st = np.zeros(4, np.uint64)
        pn = None if prev_normals is None else np.ascontiguousarray(prev_normals, np.float32)
        lib().so_trace2(self.h, _ptr(rays), rays.size, _ptr(pn), _ptr(hits), _ptr(sub),
                        _ptr(st), nthreads)
        out = [hits]
        if want_subface:
            out.append(sub)
        if want_stats:
            out.append(st)
        return out[0] if len(out) == 1 else tuple(out)

    def isect(self, rays, hits, subface=None, nthreads=0):
        """BuildIntersection's shading records (ISECT_DTYPE) of traced rays."""
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.ascontiguousarray(hits, HIT_DTYPE)
        sub = None if subface is None else np.ascontiguousarray(subface, np.uint32)
        rec = np.zeros(rays.size, ISECT_DTYPE)
        lib().so_isect_records(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(sub),
                               _ptr(rec), nthreads)
        return rec

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().so_free(self.h)
                self.h = None
        except Exception:
            pass


def canonicalize(generic_nodes, root=0):
    """Depth-first (left first) listing: (n, 10) uint32 records of leaf flag,
    axis, count, offset, bmin[3], bmax[3] bits, 0, 0."""
    g = np.ascontiguousarray(generic_nodes, NODE_DTYPE)
    out = np.zeros((g.size, 10), np.uint32)
    cnt = lib().so_canonicalize(_ptr(g), g.size, root, _ptr(out), g.size)
    if cnt < 0:
        raise ValueError("malformed tree")
    return out[:cnt]


# --------------------------------------------------------------------------
# reference accel (the real thing)
# --------------------------------------------------------------------------
DUMP_NODE_BYTES = {TRI: 64, TET: 40, SPHERE: 60}


def parse_dump(kind, data):
    """(generic nodes, sorted indices) of a file in the reference's Dump()
    format (bytes): TriangleNode 64 B, TetraNode 40 B, ParticleNode 60 B
    records, then the sorted primitive indices."""
    raw, idx = _split_dump(bytes(data), DUMP_NODE_BYTES[kind])
    if kind == TET:
        f = raw[:, :24].copy().view(np.float32).reshape(-1, 6)
        ints = raw[:, 24:40].copy().view(np.int32).reshape(-1, 4)
        g = np.zeros(raw.shape[0], NODE_DTYPE)
        g["bmin"] = f[:, :3]
        g["bmax"] = f[:, 3:]
        g["leaf"] = ints[:, 0]
        g["axis"] = np.where(ints[:, 0] == 1, 0, ints[:, 1])
        g["d0"] = ints[:, 2].view(np.uint32)
        g["d1"] = ints[:, 3].view(np.uint32)
        return g, idx
    f = raw[:, :48].copy().view(np.float32).reshape(-1, 2, 2, 3)
    slot_bmin, slot_bmax = f[:, 0], f[:, 1]
    if kind == TRI:
        ints = raw[:, 48:64].copy().view(np.int32).reshape(-1, 4)
        leaf, axis = ints[:, 0], ints[:, 1]
        d0, d1 = ints[:, 2].view(np.uint32), ints[:, 3].view(np.uint32)
    else:
        d = raw[:, 48:56].copy().view(np.uint32).reshape(-1, 2)
        sh = raw[:, 56:60].copy().view(np.int16).reshape(-1, 2)
        leaf, axis = sh[:, 0].astype(np.int32), sh[:, 1].astype(np.int32)
        d0, d1 = d[:, 0], d[:, 1]
    return generic_from_two_box(slot_bmin, slot_bmax, leaf, axis, d0, d1), idx


def _split_dump(raw, node_size):
    nn = int(np.frombuffer(raw, np.uint64, 1, 0)[0])
    nodes = np.frombuffer(raw, np.uint8, nn * node_size, 8).reshape(nn, node_size)
    off = 8 + nn * node_size
    ni = int(np.frombuffer(raw, np.uint64, 1, off)[0])
    idx = np.frombuffer(raw, np.uint32, ni, off + 8).copy()
    return nodes.copy(), idx


def _min_ref(a, b):
    """std::min(a, b) elementwise: the first operand on ties."""
    return np.where(b < a, b, a)


def _max_ref(a, b):
    return np.where(a < b, b, a)


def generic_from_device(kind, raw):
    """Device node records of libsurface_rt (srt_accel_export) -> generic
    nodes.  Two-child 64-byte nodes for triangles/spheres (leaves folded into
    the parent's child slots), own-box 32-byte nodes for tetrahedra."""
    raw = np.ascontiguousarray(raw, np.uint8)
    if kind == TET:
        f = raw.view(np.float32).reshape(-1, 8)
        u = raw.view(np.uint32).reshape(-1, 8)
        meta, ref_ = u[:, 3], u[:, 7]
        leaf = (meta & 0x80000000) != 0
        g = np.zeros(f.shape[0], NODE_DTYPE)
        g["bmin"] = f[:, 0:3]
        g["bmax"] = f[:, 4:7]
        g["leaf"] = leaf
        g["axis"] = np.where(leaf, 0, meta & 3)
        g["d0"] = np.where(leaf, meta & 0x3FFFFFFF, ref_)
        g["d1"] = np.where(leaf, ref_, ref_ + 1)
        return g
    f = raw.view(np.float32).reshape(-1, 16)
    u = raw.view(np.uint32).reshape(-1, 16)
    nb = f.shape[0]
    lo = [f[:, 0:3], f[:, 6:9]]
    hi = [f[:, 3:6], f[:, 9:12]]
    ref_ = [u[:, 12], u[:, 13]]
    cnt = [u[:, 14] & 0x3FFFFFFF, u[:, 15] & 0x3FFFFFFF]
    axis = u[:, 14] >> 30
    is_leaf = np.stack([cnt[0] > 0, cnt[1] > 0], 1)  # (nb, 2), row-major order
    nl = int(is_leaf.sum())
    leaf_id = np.full(is_leaf.shape, -1, np.int64)
    leaf_id[is_leaf] = nb + np.arange(nl)
    g = np.zeros(nb + nl, NODE_DTYPE)
    g["leaf"][:nb] = 0
    g["axis"][:nb] = axis
    child = [np.where(is_leaf[:, k], leaf_id[:, k], ref_[k]).astype(np.int64) for k in (0, 1)]
    g["d0"][:nb] = child[0]
    g["d1"][:nb] = child[1]
    for k in (0, 1):
        g["bmin"][child[k]] = lo[k]
        g["bmax"][child[k]] = hi[k]
        lk = is_leaf[:, k]
        ids = leaf_id[lk, k]
        g["leaf"][ids] = 1
        g["d0"][ids] = cnt[k][lk]
        g["d1"][ids] = ref_[k][lk]
    g["bmin"][0] = _min_ref(lo[0][0], lo[1][0])
    g["bmax"][0] = _max_ref(hi[0][0], hi[1][0])
    return g


def generic_from_two_box(slot_bmin, slot_bmax, leaf, axis, d0, d1):
    """Reference TriangleNode / ParticleNode arrays -> generic (own box) nodes.
    A branch keeps its children's boxes in slots 0/1; a leaf its own in slot 0."""
    nn = leaf.size
    g = np.zeros(nn, NODE_DTYPE)
    g["leaf"] = leaf
    g["axis"] = np.where(leaf == 1, 0, axis)
    g["d0"] = d0
    g["d1"] = d1
    br = np.nonzero(leaf == 0)[0]
    g["bmin"][d0[br]] = slot_bmin[br, 0]
    g["bmax"][d0[br]] = slot_bmax[br, 0]
    g["bmin"][d1[br]] = slot_bmin[br, 1]
    g["bmax"][d1[br]] = slot_bmax[br, 1]
    g["bmin"][0] = _min_ref(slot_bmin[0, 0], slot_bmin[0, 1])
    g["bmax"][0] = _max_ref(slot_bmax[0, 0], slot_bmax[0, 1])
    lf = np.nonzero(leaf == 1)[0]
    # a leaf's own copy must agree with its parent's slot
    if not (np.array_equal(g["bmin"][lf].view(np.uint32), slot_bmin[lf, 0].view(np.uint32))
            and np.array_equal(g["bmax"][lf].view(np.uint32), slot_bmax[lf, 0].view(np.uint32))):
        raise ValueError("leaf box differs from its parent's slot")
    return g


class RefAccel:
    """The reference's own Build32 / Traverse / Dump."""

    def __init__(self, kind, verts, faces=None, radius=None, const_radius=0.0):
        L = ref()
        if L is None:
            raise RuntimeError("reference harness not built")
        self.L = L
        self.kind = kind
        dbl = kind == TET and np.asarray(verts).dtype == np.float64
        self.verts = np.ascontiguousarray(verts, np.float64 if dbl else np.float32).reshape(-1)
        self.faces = None if faces is None else np.ascontiguousarray(faces, np.uint32).reshape(-1)
        self.radius = None if radius is None else np.ascontiguousarray(radius, np.float32)
        if kind == TRI:
            self.n = self.faces.size // 3
            self.h = L.ref_tri_build(_ptr(self.verts), self.verts.size // 3,
                                     _ptr(self.faces), self.n)
            self.tag = "tri"
        elif kind == TET:
            self.n = self.faces.size // 4
            build = L.ref_tet_build_d if dbl else L.ref_tet_build
            self.h = build(_ptr(self.verts), _ptr(self.faces), self.n)
            self.tag = "tet"
        else:
            self.n = self.verts.size // 3
            self.h = L.ref_sphere_build(_ptr(self.verts), _ptr(self.radius),
                                        C.c_float(const_radius), self.n)
            self.tag = "sphere"

    def bbox(self):
        mn = np.zeros(3)
        mx = np.zeros(3)
        getattr(self.L, f"ref_{self.tag}_bbox")(self.h, _ptr(mn), _ptr(mx))
        return mn, mx

    def dump(self):
        """(generic nodes, sorted indices) from the reference's Dump()."""
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "accel.bin")
            getattr(self.L, f"ref_{self.tag}_dump")(self.h, path.encode())
            with open(path, "rb") as fp:
                return parse_dump(self.kind, fp.read())

    def canonical(self):
        g, idx = self.dump()
        return canonicalize(g, 0), idx

    def trace(self, rays, prev_normals=None, nthreads=0, chunk=64):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        if self.kind == TRI:
            self.L.ref_tri_trace(self.h, _ptr(rays), rays.size, _ptr(hits), nthreads, chunk)
            return hits
        if self.kind == TET:
            sub = np.zeros(rays.size, np.uint32)
            self.L.ref_tet_trace(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(sub),
                                 nthreads, chunk)
            return hits, sub
        pn = None if prev_normals is None else np.ascontiguousarray(prev_normals, np.float32)
        self.L.ref_sphere_trace(self.h, _ptr(rays), rays.size, _ptr(pn), _ptr(hits),
                                nthreads, chunk)
        return hits

    def trace_isect(self, rays, prev_normals=None, nthreads=0):
        """Every Intersection field the reference's Traverse fills: (hits,
        subface (tetrahedra, else None), ISECT_DTYPE records)."""
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        rec = np.zeros(rays.size, ISECT_DTYPE)
        sub = None
        if self.kind == TRI:
            self.L.ref_tri_trace_isect(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(rec),
                                       nthreads)
        elif self.kind == TET:
            sub = np.zeros(rays.size, np.uint32)
            self.L.ref_tet_trace_isect(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(sub),
                                       _ptr(rec), nthreads)
        else:
            pn = None if prev_normals is None else np.ascontiguousarray(prev_normals,
                                                                        np.float32)
            self.L.ref_sphere_trace_isect(self.h, _ptr(rays), rays.size, _ptr(pn), _ptr(hits),
                                          _ptr(rec), nthreads)
        return hits, sub, rec

    def __del__(self):
        try:
            if getattr(self, "h", None):
                getattr(self.L, f"ref_{self.tag}_free")(self.h)
                self.h = None
        except Exception:
            pass


# --------------------------------------------------------------------------
# stage-level helpers
# --------------------------------------------------------------------------
def tinymt64_doubles(n, seed=123456, use_ref=False):
    out = np.zeros(n, np.float64)
    if use_ref:
        ref().ref_tinymt64_doubles(seed, TMT_MAT1, TMT_MAT2, TMT_TMAT, n, _ptr(out))
    else:
        lib().so_tinymt64_doubles(seed, TMT_MAT1, TMT_MAT2, TMT_TMAT, n, _ptr(out))
    return out


def fixture_points(n, rng_state=None, seed=123456):
    """The reference tests' point draws: (float)genrand_double() x 3 per point."""
    d = tinymt64_doubles(3 * n, seed)
    return d.astype(np.float32).reshape(n, 3)


def morton_points(pts, bmin, bmax):
    pts = np.ascontiguousarray(pts, np.float32)
    out = np.zeros(pts.size // 3, np.uint32)
    lib().so_morton_points(_ptr(pts), out.size, _ptr(np.asarray(bmin, np.float32)),
                           _ptr(np.asarray(bmax, np.float32)), _ptr(out))
    return out


def sort_pairs(codes, index=None):
    c = np.ascontiguousarray(codes, np.uint32).copy()
    i = (np.arange(c.size, dtype=np.uint32) if index is None
         else np.ascontiguousarray(index, np.uint32).copy())
    lib().so_sort_pairs(_ptr(c), _ptr(i), c.size)
    return c, i


def karras(sorted_codes):
    c = np.ascontiguousarray(sorted_codes, np.uint32)
    m = c.size - 1
    child = np.zeros(m, np.uint32)
    lt = np.zeros(m, np.uint8)
    rt = np.zeros(m, np.uint8)
    lib().so_karras(_ptr(c), c.size, _ptr(child), _ptr(lt), _ptr(rt))
    return child, lt, rt


def tex3d(img, dims, uvw, clamp=(1, 1, 1)):
    img = np.ascontiguousarray(img, np.float32)
    uvw = np.ascontiguousarray(uvw, np.float32)
    out = np.zeros(uvw.size // 3, np.float32)
    d = np.asarray(dims, np.int32)
    lib().so_tex3d(_ptr(img), _ptr(d), _ptr(uvw), out.size, *clamp, _ptr(out))
    return out


# volume parameters (so_vol_params)
VOL_DTYPE = np.dtype([("width", "<i4"), ("height", "<i4"), ("max_steps", "<i4"),
                      ("reserved", "<i4"), ("eye", "<f4", 3), ("corner", "<f4", 3),
                      ("du", "<f4", 3), ("dv", "<f4", 3), ("step", "<f4"),
                      ("sigma_scale", "<f4"), ("alpha_max", "<f4")])


def volume_params(width, height, eye, lookat, up, fov_deg, step, sigma_scale,
                  alpha_max, max_steps):
    p = np.zeros(1, VOL_DTYPE)
    p["width"], p["height"], p["max_steps"] = width, height, max_steps
    corner = np.zeros(3, np.float32)
    du = np.zeros(3, np.float32)
    dv = np.zeros(3, np.float32)
    e = np.asarray(eye, np.float32)
    lib().so_volume_camera(width, height, _ptr(e), _ptr(np.asarray(lookat, np.float32)),
                           _ptr(np.asarray(up, np.float32)), C.c_float(fov_deg),
                           _ptr(corner), _ptr(du), _ptr(dv))
    p["eye"], p["corner"], p["du"], p["dv"] = e, corner, du, dv
    p["step"], p["sigma_scale"], p["alpha_max"] = step, sigma_scale, alpha_max
    return p


class _Sampling(C.Structure):
    _fields_ = [("remap", C.c_void_p * 3), ("remap_n", C.c_uint32 * 3),
                ("clamp", C.c_int32 * 3)]


def _sampling(remap, clamp):
    """so_sampling for remap tables (None each) and clamp flags, or None for
    the default (clamp-to-edge, no remap); the tables are kept alive on it."""
    if remap is None and clamp is None:
        return None
    sm = _Sampling()
    remap = remap or (None, None, None)
    clamp = (1, 1, 1) if clamp is None else clamp
    sm.keep = [None if t is None else np.ascontiguousarray(t, np.float32) for t in remap]
    for k in range(3):
        t = sm.keep[k]
        sm.remap[k] = None if t is None else t.ctypes.data
        sm.remap_n[k] = 0 if t is None else t.size
        sm.clamp[k] = int(clamp[k])
    return sm


def volume_fwd_f32(params, dens, dims, tf, nthreads=0, remap=None, clamp=None):
    """FP32 march; remap (3 tables or None) and clamp (3 flags) give the
    density texture's sampling state (default: clamp-to-edge, no remap)."""
    W, H = int(params["width"][0]), int(params["height"][0])
    img = np.zeros((H, W, 4), np.float32)
    sm = _sampling(remap, clamp)
    lib().so_volume_fwd_f32_ex(_ptr(params), None if sm is None else C.byref(sm),
                               _ptr(np.ascontiguousarray(dens, np.float32)),
                               _ptr(np.asarray(dims, np.int32)),
                               _ptr(np.ascontiguousarray(tf, np.float32)), _ptr(img), nthreads)
    return img


def volume_f64(params, dens, dims, tf, target=None, want_grad=False, want_img=False,
               remap=None, clamp=None):
    W, H = int(params["width"][0]), int(params["height"][0])
    dens = np.ascontiguousarray(dens, np.float64)
    tf = np.ascontiguousarray(tf, np.float64)
    img = np.zeros((H, W, 4)) if want_img else None
    gd = np.zeros(dens.shape) if want_grad else None
    gt = np.zeros(tf.shape) if want_grad else None
    tg = None if target is None else np.ascontiguousarray(target, np.float32)
    sm = _sampling(remap, clamp)
    loss = lib().so_volume_f64_ex(_ptr(params), None if sm is None else C.byref(sm),
                                  _ptr(dens), _ptr(np.asarray(dims, np.int32)), _ptr(tf),
                                  _ptr(tg), _ptr(img), _ptr(gd), _ptr(gt))
    return loss, img, gd, gt


def volume_f64_pixels(params, dens, dims, tf, target, pixels):
    """The FP64 loss over the listed pixels (py * width + px) only."""
    dens = np.ascontiguousarray(dens, np.float64)
    tf = np.ascontiguousarray(tf, np.float64)
    tg = np.ascontiguousarray(target, np.float32)
    px = np.ascontiguousarray(pixels, np.uint32)
    return lib().so_volume_f64_pixels(_ptr(params), _ptr(dens),
                                      _ptr(np.asarray(dims, np.int32)), _ptr(tf), _ptr(tg),
                                      _ptr(px), px.size)


def volume_pixels_near(params, dims, center, radius):
    """Pixels whose rays pass within `radius` texels (max norm) of texel
    `center` (x, y, z) of a uniform volume: the only ones a change of that
    texel can affect (a conservative superset, from the rays' slab entry and
    exit in float64)."""
    W, H = int(params["width"][0]), int(params["height"][0])
    px, py = np.meshgrid(np.arange(W) + 0.5, np.arange(H) + 0.5)
    v = (params["corner"][0][None, None, :] + px[..., None] * params["du"][0]
         + py[..., None] * params["dv"][0] - params["eye"][0])
    d = v / np.linalg.norm(v, axis=-1, keepdims=True)
    o = params["eye"][0].astype(np.float64)
    # texel i of n spans world [2 i/(n-1) - 1 +- 2 r/(n-1)] (texel-corner map u = 0.5 p + 0.5)
    lo = np.array([2.0 * (center[k] - radius) / (dims[k] - 1) - 1.0 for k in range(3)])
    hi = np.array([2.0 * (center[k] + radius) / (dims[k] - 1) - 1.0 for k in range(3)])
    with np.errstate(divide="ignore", invalid="ignore"):
        ta = (lo - o) / d
        tb = (hi - o) / d
    tmin = np.nanmax(np.minimum(ta, tb), axis=-1)
    tmax = np.nanmin(np.maximum(ta, tb), axis=-1)
    hit = tmin <= tmax
    return np.nonzero(hit.reshape(-1))[0].astype(np.uint32)


# ---------------------------------------------------------------- eye rays
def camera_frame(eye, lookat, up, fov, ortho, width, height, use_ref=False):
    """(corner, u, v) of Camera::buildFrame -- the restatement, or with
    use_ref the reference's own (render/render_camera.cc:17-63)."""
    e, la, u = (np.ascontiguousarray(x, np.float32) for x in (eye, lookat, up))
    out = np.zeros(9, np.float32)
    L = ref() if use_ref else lib()
    fn = L.ref_camera_frame if use_ref else L.so_camera_frame
    fn(_ptr(e), _ptr(la), _ptr(u), C.c_float(fov), int(ortho), int(width), int(height),
       _ptr(out))
    return out[:3], out[3:6], out[6:]


def camera_rays(cam):
    """OnData's eye rays for one sample per pixel (see so_camera_rays).
    cam: dict with eye, lookat, up, fov, ortho, width, height, viewport
    (x, y, w, h), region (x0, y0, x1, y1), step.  Returns (rays, pixel)."""
    f = np.zeros(10, np.float32)
    f[0:3], f[3:6], f[6:9], f[9] = cam["eye"], cam["lookat"], cam["up"], cam["fov"]
    ints = np.array([cam["ortho"], cam["width"], cam["height"], *cam["viewport"],
                     *cam["region"], cam["step"]], np.int32)
    x0, y0, x1, y1 = cam["region"]
    cap = max(1, len(range(x0, x1, cam["step"])) * len(range(y0, y1, cam["step"])))
    rays = np.zeros(cap, RAY_DTYPE)
    pix = np.zeros(cap, np.uint32)
    n = lib().so_camera_rays(_ptr(f), _ptr(ints), _ptr(rays), _ptr(pix))
    return rays[:n], pix[:n]


def stereo_env_ray(eye, lookat, up, zero_parallax, eye_separation, image_u, image_v, width,
                   height, use_ref=False):
    """Camera::generateStereoEnvRay -- the restatement, or with use_ref the
    reference's own (render/render_camera.cc:65-118).  Returns (org, dir)."""
    e, la, u = (np.ascontiguousarray(x, np.float32) for x in (eye, lookat, up))
    if use_ref:
        out = np.zeros(6, np.float32)
        ref().ref_stereo_env_ray(_ptr(e), _ptr(la), _ptr(u), C.c_float(zero_parallax),
                                 C.c_float(eye_separation), C.c_float(image_u),
                                 C.c_float(image_v), int(width), int(height), _ptr(out))
        return out[:3], out[3:]
    o = np.zeros(3, np.float32)
    d = np.zeros(3, np.float32)
    lib().so_stereo_env_ray(_ptr(e), _ptr(la), _ptr(u), C.c_float(zero_parallax),
                            C.c_float(eye_separation), C.c_float(image_u), C.c_float(image_v),
                            int(width), int(height), _ptr(o), _ptr(d))
    return o, d


def camera_rays_ex(cam, subsamples=1, stereo=None, seed=1234, offset=0):
    """OnData's eye rays with subsamples x subsamples rays per pixel (the
    serial renderer's jitter stream: TinyMT64 seeded `seed`, `offset` draws
    consumed before the frame) and, with stereo = (zero_parallax,
    eye_separation), the stereo environment camera.  Returns (rays, pixel),
    subsamples^2 consecutive rays per kept loop pixel."""
    f = np.zeros(10, np.float32)
    f[0:3], f[3:6], f[6:9], f[9] = cam["eye"], cam["lookat"], cam["up"], cam["fov"]
    ints = np.array([cam["ortho"], cam["width"], cam["height"], *cam["viewport"],
                     *cam["region"], cam["step"]], np.int32)
    si = np.array([subsamples, 1 if stereo else 0], np.int32)
    sf = np.array(stereo if stereo else (0.0, 0.0), np.float32)
    x0, y0, x1, y1 = cam["region"]
    cap = max(1, len(range(x0, x1, cam["step"])) * len(range(y0, y1, cam["step"])))
    cap *= subsamples * subsamples
    rays = np.zeros(cap, RAY_DTYPE)
    pix = np.zeros(cap, np.uint32)
    n = lib().so_camera_rays_ex(_ptr(f), _ptr(ints), _ptr(si), _ptr(sf), C.c_uint64(seed),
                                C.c_uint64(offset), _ptr(rays), _ptr(pix))
    return rays[:n], pix[:n]


def framebuffer_write_ex(cam, subsamples, hits, pixel, rgba=None, fmt=0, color=None,
                         depth=None):
    """The write of camera_rays_ex's rays: each pixel's hits averaged."""
    W, H = cam["width"], cam["height"]
    if color is None:
        color = np.zeros((H, W, 4), np.uint8 if fmt == 0 else np.float32)
    if depth is None:
        depth = np.zeros((H, W), np.float32)
    hits = np.ascontiguousarray(hits, HIT_DTYPE)
    pixel = np.ascontiguousarray(pixel, np.uint32)
    rg = None if rgba is None else np.ascontiguousarray(rgba, np.float32)
    lib().so_framebuffer_write_ex(W, H, cam["step"], int(subsamples), _ptr(hits), _ptr(pixel),
                                  None if rg is None else _ptr(rg), hits.size, fmt,
                                  _ptr(color), _ptr(depth))
    return color, depth


def framebuffer_write(cam, hits, pixel, rgba=None, fmt=0, color=None, depth=None):
    """OnData's write of the hit rays into (color, depth); color RGBA8
    (fmt 0, uint8 (H, W, 4)) or RGBA32F (fmt 1, float32 (H, W, 4))."""
    W, H = cam["width"], cam["height"]
    if color is None:
        color = np.zeros((H, W, 4), np.uint8 if fmt == 0 else np.float32)
    if depth is None:
        depth = np.zeros((H, W), np.float32)
    hits = np.ascontiguousarray(hits, HIT_DTYPE)
    pixel = np.ascontiguousarray(pixel, np.uint32)
    rg = None if rgba is None else np.ascontiguousarray(rgba, np.float32)
    lib().so_framebuffer_write(W, H, cam["step"], _ptr(hits), _ptr(pixel),
                               None if rg is None else _ptr(rg), hits.size, fmt,
                               _ptr(color), _ptr(depth))
    return color, depth


# ------------------------------------------------------------------- scenes
def _top_arrays(fn, h, cap):
    boxes = np.zeros((cap, 6), np.float64)
    ints = np.zeros((cap, 5), np.int32)
    n = fn(h, _ptr(boxes), _ptr(ints), cap)
    return boxes[:n].copy(), ints[:n].copy()


def matrix_inverse(m, use_ref=False):
    """Matrixd::Inverse of a row-major 4x4: the restatement, or with use_ref
    the reference's own."""
    a = np.array(m, np.float64).reshape(16).copy()
    (ref().ref_matrix_inverse if use_ref else lib().so_matrix_inverse)(_ptr(a))
    return a.reshape(4, 4)


def element_update(T, lbmin, lbmax):
    """RenderElement::Update: (invT, invT33, world bmin, world bmax)."""
    T = np.ascontiguousarray(T, np.float64).reshape(16)
    lo = np.ascontiguousarray(lbmin, np.float64)
    hi = np.ascontiguousarray(lbmax, np.float64)
    iT, iT33 = np.zeros(16), np.zeros(16)
    wlo, whi = np.zeros(3), np.zeros(3)
    lib().so_element_update(_ptr(T), _ptr(lo), _ptr(hi), _ptr(iT), _ptr(iT33), _ptr(wlo),
                            _ptr(whi))
    return iT.reshape(4, 4), iT33.reshape(4, 4), wlo, whi


class RefTopTree:
    """The reference's own BVHTree (render/render_bvh_tree.cc) over world
    boxes: node arrays and per-ray candidate lists."""

    def __init__(self, bmin, bmax, ids=None):
        self.bmin = np.ascontiguousarray(bmin, np.float64).reshape(-1, 3)
        self.bmax = np.ascontiguousarray(bmax, np.float64).reshape(-1, 3)
        n = self.bmin.shape[0]
        self.ids = (np.arange(n, dtype=np.uint32) if ids is None
                    else np.ascontiguousarray(ids, np.uint32))
        self.h = ref().ref_bvh_build(_ptr(self.bmin), _ptr(self.bmax), _ptr(self.ids), n)
        self.cap = 2 * n + 2

    def nodes(self):
        return _top_arrays(ref().ref_bvh_nodes, self.h, self.cap)

    def candidates(self, org, dir_):
        o = np.ascontiguousarray(org, np.float64)
        d = np.ascontiguousarray(dir_, np.float64)
        cap = self.bmin.shape[0] + 1
        tt = np.zeros((cap, 2), np.float64)
        ids = np.zeros(cap, np.uint32)
        n = ref().ref_bvh_trace(self.h, _ptr(o), _ptr(d), _ptr(tt), _ptr(ids), cap)
        return tt[:n, 0].copy(), ids[:n].copy()

    def __del__(self):
        try:
            if getattr(self, "h", None):
                ref().ref_bvh_free(self.h)
                self.h = None
        except Exception:
            pass


class OracleScene:
    """RenderGraph::Build / Trace restated (so_scene_*): elements are
    OracleAccel, OracleLines or OracleSolids objects with their transforms
    (4x4 row-major doubles as Matrixd's m[row][col]) and world boxes."""

    def __init__(self, accels, T, invT, invT33, bmin, bmax):
        self.accels = list(accels)  # None entries: top-level tree only
        n = len(self.accels)
        self._T = np.ascontiguousarray(T, np.float64).reshape(n, 16)
        self._iT = np.ascontiguousarray(invT, np.float64).reshape(n, 16)
        self._iT33 = np.ascontiguousarray(invT33, np.float64).reshape(n, 16)
        self._bmin = np.ascontiguousarray(bmin, np.float64).reshape(n, 3)
        self._bmax = np.ascontiguousarray(bmax, np.float64).reshape(n, 3)
        hs = (C.c_void_p * n)(*[None if a is None else a.h for a in self.accels])
        self.h = lib().so_scene_build(hs, _ptr(self._T), _ptr(self._iT), _ptr(self._iT33),
                                      _ptr(self._bmin), _ptr(self._bmax), n)
        for e, a in enumerate(self.accels):
            if isinstance(a, (OracleLines, OracleSolids)):
                lib().so_scene_set_kind(self.h, e, 3 if isinstance(a, OracleLines) else 4)
        self.cap = 2 * n + 2

    def nodes(self):
        return _top_arrays(lib().so_scene_top_nodes, self.h, self.cap)

    def candidates(self, org, dir_):
        o = np.ascontiguousarray(org, np.float64)
        d = np.ascontiguousarray(dir_, np.float64)
        cap = len(self.accels) + 1
        tt = np.zeros(cap, np.float64)
        ids = np.zeros(cap, np.uint32)
        n = lib().so_scene_candidates(self.h, _ptr(o), _ptr(d), _ptr(tt), _ptr(ids), cap)
        return tt[:n].copy(), ids[:n].copy()

    def trace(self, rays, prev_element=None, prev_normals=None, nthreads=0,
              want_visits=False, walk2=False):
        """(hits, element): hit t is the world distance, prim / u / v the
        element's own; element MISS where nothing was hit.  want_visits adds
        per-ray node + primitive visits of the element walks; walk2 walks the
        elements with the two-pass walk restated instead of the reference's."""
        if any(a is None for a in self.accels):
            raise ValueError("scene built without accels")
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        el = np.zeros(rays.size, np.uint32)
        pe = None if prev_element is None else np.ascontiguousarray(prev_element, np.uint32)
        pn = None if prev_normals is None else np.ascontiguousarray(prev_normals, np.float32)
        vis = np.zeros(rays.size, np.uint32) if want_visits else None
        lib().so_scene_trace(self.h, _ptr(rays), rays.size, _ptr(pe), _ptr(pn), _ptr(hits),
                             _ptr(el), _ptr(vis), 1 if walk2 else 0, nthreads)
        return (hits, el, vis) if want_visits else (hits, el)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().so_scene_free(self.h)
                self.h = None
        except Exception:
            pass


# ---------------------------------------------------------- texture fetch
TEX_FORMATS = {0: np.uint8, 1: np.float32, 2: np.float64}
BLOCK_DTYPE = np.dtype([("offset", "<i4", 3), ("extent", "<i4", 3), ("size", "<i4", 3),
                        ("level", "<i4"), ("data_offset", "<u8")])


def tex_fetch(fmt, img, comps, uvw, clamp=(1, 1, 1), remap=(None, None, None), use_ref=False):
    """Texture::Fetch of a dense 3D texture img (D, H, W[, comps]) of format
    fmt (0 byte, 1 float, 2 double): (n, 4) float32."""
    img = np.ascontiguousarray(img, TEX_FORMATS[fmt])
    d, h, w = img.shape[:3]
    uvw = np.ascontiguousarray(uvw, np.float32).reshape(-1, 3)
    out = np.zeros((uvw.shape[0], 4), np.float32)
    cl = np.ascontiguousarray(clamp, np.int32)
    tabs = [None if t is None else np.ascontiguousarray(t, np.float32) for t in remap]
    ns = [0 if t is None else t.size for t in tabs]
    if use_ref:
        ref().ref_tex_fetch(fmt, _ptr(img), w, h, d, comps, _ptr(cl), _ptr(tabs[0]), ns[0],
                            _ptr(tabs[1]), ns[1], _ptr(tabs[2]), ns[2], _ptr(uvw),
                            uvw.shape[0], _ptr(out))
    else:
        dim = np.array([w, h, d], np.int32)
        tp = (C.c_void_p * 3)(*[None if t is None else t.ctypes.data for t in tabs])
        npa = np.array(ns, np.int32)
        lib().so_tex_fetch(fmt, _ptr(img), _ptr(dim), comps, _ptr(cl), tp, _ptr(npa),
                           _ptr(uvw), uvw.shape[0], _ptr(out))
    return out


def sparse_fetch(blocks, pool, fmt, comps, gdim, uvw, use_ref=False):
    """Texture::Fetch of a sparse volume: blocks (BLOCK_DTYPE), pool (bytes
    of every block's voxels at data_offset): (n, 4) float32."""
    blocks = np.ascontiguousarray(blocks, BLOCK_DTYPE)
    pool = np.ascontiguousarray(np.frombuffer(bytes(pool), np.uint8))
    g = np.ascontiguousarray(gdim, np.int32)
    uvw = np.ascontiguousarray(uvw, np.float32).reshape(-1, 3)
    out = np.zeros((uvw.shape[0], 4), np.float32)
    if use_ref:
        ref().ref_sparse_fetch(_ptr(blocks), blocks.size, _ptr(pool), fmt, comps, _ptr(g),
                               _ptr(uvw), uvw.shape[0], _ptr(out))
    else:
        tree = lib().so_sparse_tree(_ptr(blocks), blocks.size)
        try:
            lib().so_sparse_fetch(tree, _ptr(blocks), _ptr(pool), fmt, comps, _ptr(g),
                                  _ptr(uvw), uvw.shape[0], _ptr(out))
        finally:
            lib().so_scene_free(tree)
    return out


# ---------------------------------------------------------------- lines
LINE_NODE_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("flag", "<i4"),
                            ("axis", "<i4"), ("data", "<u4", 2)])  # LineNode, 40 bytes


def parse_line_dump(raw):
    """LineAccel::Dump(): (nodes LINE_NODE_DTYPE, indices uint32)."""
    nn = int(np.frombuffer(raw[:8], np.uint64)[0])
    nodes = np.frombuffer(raw[8:8 + 40 * nn], LINE_NODE_DTYPE).copy()
    off = 8 + 40 * nn
    ni = int(np.frombuffer(raw[off:off + 8], np.uint64)[0])
    idx = np.frombuffer(raw[off + 8:off + 8 + 4 * ni], np.uint32).copy()
    return nodes, idx


def line_nodes_masked(nodes):
    """Node records with the fields a leaf leaves unset (its axis) zeroed."""
    n = nodes.copy()
    n["axis"][n["flag"] == 1] = 0
    return n


class _LinesBase:
    def _inputs(self, pos, segments, radius, const_radius):
        self.pos = np.ascontiguousarray(pos, np.float32).reshape(-1)
        self.seg = np.ascontiguousarray(segments, np.uint32).reshape(-1)
        self.radius = None if radius is None else np.ascontiguousarray(radius, np.float32)
        self.const_radius = float(const_radius)
        self.n = self.seg.size // 2


class OracleLines(_LinesBase):
    """The restatement of LineAccel: Build, Traverse (hits and normals)."""

    def __init__(self, pos, segments, radius=None, const_radius=0.0, min_leaf=4,
                 max_depth=512, cap=True):
        self._inputs(pos, segments, radius, const_radius)
        self.h = lib().so_line_build(_ptr(self.pos), _ptr(self.radius),
                                     C.c_float(self.const_radius), _ptr(self.seg), self.n,
                                     min_leaf, max_depth, int(cap))

    def export(self):
        nn = lib().so_line_num_nodes(self.h)
        nodes = np.zeros(nn, LINE_NODE_DTYPE)
        idx = np.zeros(self.n, np.uint32)
        lib().so_line_export(self.h, _ptr(nodes), _ptr(idx))
        return nodes, idx

    def depth(self):
        return lib().so_line_depth(self.h)

    def trace(self, rays, nthreads=0):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        nrm = np.zeros((rays.size, 3), np.float32)
        lib().so_line_trace(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(nrm), nthreads)
        return hits, nrm

    def __del__(self):
        try:
            lib().so_line_free(self.h)
        except Exception:  # noqa: BLE001
            pass


class RefLines(_LinesBase):
    """The reference's own LineAccel (Build, Traverse, Dump, BoundingBox)."""

    def __init__(self, pos, segments, radius=None, const_radius=0.0, min_leaf=4,
                 max_depth=512, cap=True):
        L = ref()
        if L is None:
            raise RuntimeError("reference harness not built")
        self.L = L
        self._inputs(pos, segments, radius, const_radius)
        self.h = L.ref_line_build(_ptr(self.pos), _ptr(self.radius),
                                  C.c_float(self.const_radius), _ptr(self.seg), self.n,
                                  min_leaf, max_depth, int(cap))

    def dump_bytes(self):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "lines.bin")
            self.L.ref_line_dump(self.h, path.encode())
            with open(path, "rb") as fp:
                return fp.read()

    def dump(self):
        return parse_line_dump(self.dump_bytes())

    def bbox(self):
        mn = np.zeros(3)
        mx = np.zeros(3)
        self.L.ref_line_bbox(self.h, _ptr(mn), _ptr(mx))
        return mn, mx

    def trace(self, rays, nthreads=0, chunk=64):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        nrm = np.zeros((rays.size, 3), np.float32)
        self.L.ref_line_trace(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(nrm),
                              nthreads, chunk)
        return hits, nrm

    def __del__(self):
        try:
            self.L.ref_line_free(self.h)
        except Exception:  # noqa: BLE001
            pass


# ---------------------------------------------------------------- solids
SOLID_NODE_DTYPE = LINE_NODE_DTYPE  # SolidNode: the same 40-byte record


def parse_solid_dump(raw):
    """SolidAccel::Dump(): (nodes SOLID_NODE_DTYPE, indices uint32)."""
    return parse_line_dump(raw)


def _solid_verts(verts):
    """float64 vertices keep double precision (Solid::dvertices); any other
    dtype is taken as float32."""
    v = np.asarray(verts)
    dt = np.float64 if v.dtype == np.float64 else np.float32
    return np.ascontiguousarray(v, dt).reshape(-1)


class OracleSolids:
    """The restatement of SolidAccel::Build32 / Traverse (nv = 5 pyramids,
    6 prisms, 8 hexahedra); float64 vertices are double-precision positions."""

    def __init__(self, nv, verts, indices, sah=False):
        """sah: SolidAccel::Build (binned SAH) at every size."""
        self.nv = int(nv)
        self.verts = _solid_verts(verts)
        self.ix = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        self.n = self.ix.size // self.nv
        dbl = self.verts.dtype == np.float64
        if sah:
            self.h = lib().so_solid_build_sah(self.nv, None if dbl else _ptr(self.verts),
                                              _ptr(self.verts) if dbl else None, _ptr(self.ix),
                                              self.n)
        else:
            build = lib().so_solid_build_d if dbl else lib().so_solid_build
            self.h = build(self.nv, _ptr(self.verts), _ptr(self.ix), self.n)

    def export(self):
        nn = lib().so_solid_num_nodes(self.h)
        nodes = np.zeros(nn, SOLID_NODE_DTYPE)
        idx = np.zeros(self.n, np.uint32)
        lib().so_solid_export(self.h, _ptr(nodes), _ptr(idx))
        return nodes, idx

    def trace(self, rays, nthreads=0):
        """(hits, normals, positions)."""
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        nrm = np.zeros((rays.size, 3), np.float32)
        pos = np.zeros((rays.size, 3), np.float32)
        lib().so_solid_trace(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(nrm), _ptr(pos),
                             nthreads)
        return hits, nrm, pos

    def __del__(self):
        try:
            lib().so_solid_free(self.h)
        except Exception:  # noqa: BLE001
            pass


class RefSolids:
    """The reference's own SolidAccel (Build32, Traverse, Dump, BoundingBox)."""

    def __init__(self, nv, verts, indices, sah=False):
        """sah: SolidAccel::Build (binned SAH) at every size."""
        L = ref()
        if L is None:
            raise RuntimeError("reference harness not built")
        self.L = L
        self.nv = int(nv)
        self.verts = _solid_verts(verts)
        self.ix = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        self.n = self.ix.size // self.nv
        dbl = self.verts.dtype == np.float64
        if sah:
            self.h = L.ref_solid_build_sah(self.nv, None if dbl else _ptr(self.verts),
                                           _ptr(self.verts) if dbl else None, _ptr(self.ix),
                                           self.n)
        else:
            build = L.ref_solid_build_d if dbl else L.ref_solid_build
            self.h = build(self.nv, _ptr(self.verts), _ptr(self.ix), self.n)

    def dump(self):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "solids.bin")
            self.L.ref_solid_dump(self.h, path.encode())
            with open(path, "rb") as fp:
                return parse_solid_dump(fp.read())

    def bbox(self):
        mn = np.zeros(3)
        mx = np.zeros(3)
        self.L.ref_solid_bbox(self.h, _ptr(mn), _ptr(mx))
        return mn, mx

    def trace(self, rays, nthreads=0, chunk=64):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(rays.size, HIT_DTYPE)
        nrm = np.zeros((rays.size, 3), np.float32)
        pos = np.zeros((rays.size, 3), np.float32)
        self.L.ref_solid_trace(self.h, _ptr(rays), rays.size, _ptr(hits), _ptr(nrm), _ptr(pos),
                               nthreads, chunk)
        return hits, nrm, pos

    def __del__(self):
        try:
            self.L.ref_solid_free(self.h)
        except Exception:  # noqa: BLE001
            pass


def tree_canonical(nodes, root=0):
    """A 40-byte-node tree (LineNode / SolidNode) as a pre-order list of its
    nodes from the root, independent of the record order: branches (axis,
    box) and leaves (box, count, first)."""
    out, stack = [], [root]
    while stack:
        nd = nodes[stack.pop()]
        if nd["flag"] == 1:
            out.append(("L", nd["bmin"].tobytes(), nd["bmax"].tobytes(), int(nd["data"][0]),
                        int(nd["data"][1])))
        else:
            out.append(("B", int(nd["axis"]), nd["bmin"].tobytes(), nd["bmax"].tobytes()))
            stack.append(int(nd["data"][1]))
            stack.append(int(nd["data"][0]))
    return out
