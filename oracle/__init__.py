"""CPU checkers for the SVBRDF fitting path.  TEST INFRASTRUCTURE ONLY.

Two libraries sit behind this module, both built by ``oracle/Makefile``:

* ``libsvf_oracle.so`` -- the C restatement of the reference path
  (``svf_oracle.c``); always available.
* ``_ref/libtempest_ref.so`` -- the reference's own CPU fitter compiled from its
  sources with ``ref_harness.cc``; available where it was built.

Only tests, ``bench.py``'s CPU-baseline leg and ``__graft_entry__.smoke()`` use
them, as checkers or as the timed CPU baseline.  The product package
(``tempestrenderer_b200``) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libsvf_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtempest_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


def build(reference_root: str | None = None) -> None:
    """Builds the restatement and, when the reference sources exist, the reference."""
    args = ["make", "-s", "-C", HERE, "-j8", "all"]
    if reference_root:
        args.append(f"REFERENCE_ROOT={reference_root}")
    subprocess.run(args, check=True)


# ----------------------------------------------------------------------------
# the C restatement
# ----------------------------------------------------------------------------


class LsqStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("effective", C.c_uint32),
                ("jacobians", C.c_uint32), ("residuals", C.c_uint32), ("mse", C.c_double)]


class Mesh(C.Structure):
    _fields_ = [("lights_parabolic", C.c_void_p), ("light_count", C.c_uint32),
                ("triangles", C.c_void_p), ("triangle_count", C.c_uint32),
                ("edges", C.c_void_p), ("edge_angles", C.c_void_p), ("edge_count", C.c_uint32)]


class InitInfo(C.Structure):
    _fields_ = [("ndf_denom", C.c_float), ("normal", C.c_float * 3), ("tangent", C.c_float * 3),
                ("basis", C.c_float * 9), ("sggx_stddev", C.c_float * 3)]


class Truth(C.Structure):
    _fields_ = [("kd", C.c_float * 3), ("ks", C.c_float * 3), ("sigma", C.c_float * 2),
                ("quat", C.c_float * 4), ("euler", C.c_float * 3), ("kind", C.c_uint32)]


_oracle = None


def lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.svfo_ring81_angles.argtypes = [_f32p]
        L.svfo_ring81_angles.restype = C.c_uint32
        L.svfo_angles_to_parabolic.argtypes = [_f32p, C.c_uint32, _f32p]
        L.svfo_brdf_f32.argtypes = [_f64p, _f32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float]
        L.svfo_brdf_f32.restype = C.c_float
        L.svfo_brdf_f64.argtypes = [_f64p, _f32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double]
        L.svfo_brdf_f64.restype = C.c_double
        L.svfo_brdf_eval_all.argtypes = [_f64p, _f32p, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p]
        L.svfo_brdf_ms_eval_all.argtypes = [_f64p, _f32p, C.c_uint32, C.c_uint32, _f32p]
        L.svfo_pseudo_volume_rgb.argtypes = [_f32p, _f32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                             C.c_uint32, _f32p]
        L.svfo_lsq_fit.argtypes = [_f32p, _f32p, C.c_uint32, C.c_float, C.c_uint32, _f32p, _f32p,
                                   C.POINTER(LsqStats)]
        L.svfo_lsq_fit.restype = C.c_float
        L.svfo_lsq_fit_ms.argtypes = [_f32p, _f32p, C.c_uint32, C.c_uint32, C.c_uint32, _f32p, _f32p,
                                      C.POINTER(LsqStats)]
        L.svfo_lsq_fit_ms.restype = C.c_float
        L.svfo_lum_slice.argtypes = [_f32p, C.c_uint32, _f32p, _f32p]
        L.svfo_sample_lum.argtypes = [C.POINTER(Mesh), _f32p, _f32p, _f32p]
        L.svfo_sample_lum.restype = C.c_float
        L.svfo_ndf_texture.argtypes = [C.POINTER(Mesh), _f32p, _f32p]
        L.svfo_ndf_sample.argtypes = [_f32p, C.c_float, C.c_float]
        L.svfo_ndf_sample.restype = C.c_float
        L.svfo_default_init_from_ndf.argtypes = [_f32p, _f32p, C.POINTER(InitInfo)]
        L.svfo_decompose.argtypes = [_f32p, _f32p, _f32p]
        L.svfo_euler_to_matrix.argtypes = [_f32p, C.c_void_p, C.c_void_p]
        L.svfo_philox4x32.argtypes = [_u32p, _u32p, _u32p]
        L.svfo_synth_truth.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(Truth)]
        L.svfo_synth_render.argtypes = [C.c_uint32, C.c_uint64, C.POINTER(Truth), _f32p, C.c_uint32,
                                        C.c_float, _f32p]
        L.svfo_btf_decode.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p]
        _oracle = L
    return _oracle


def ring81_angles() -> np.ndarray:
    out = np.zeros((81, 2), np.float32)
    n = lib().svfo_ring81_angles(out)
    assert n == 81
    return out


def angles_to_parabolic(theta_phi: np.ndarray) -> np.ndarray:
    tp = np.ascontiguousarray(theta_phi, np.float32)
    out = np.zeros_like(tp)
    lib().svfo_angles_to_parabolic(tp, tp.shape[0], out)
    return out


def brdf_all(params7, lights_parabolic, fresnel=1.0):
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    L = lp.shape[0]
    p = np.ascontiguousarray(params7, np.float64)
    f32 = np.zeros(L * L, np.float32)
    f64 = np.zeros(L * L, np.float64)
    lib().svfo_brdf_eval_all(p, lp, L, fresnel, f32.ctypes.data, f64.ctypes.data)
    return f32, f64


def brdf_all_ms(params7, lights_parabolic, bounces):
    """The fitter's pseudo-volume (multi-scattering) BRDF over all pairs (FP32, the
    reference's operation order and random sequence)."""
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    L = lp.shape[0]
    out = np.zeros(L * L, np.float32)
    lib().svfo_brdf_ms_eval_all(np.ascontiguousarray(params7, np.float64), lp, L, bounces, out)
    return out


def pseudo_volume_rgb(params_rgb, lights_parabolic, view, light, bounces, samples=256, seed=0):
    """The pseudo-volume BRDF of one material (sx, sy, quaternion xyzw, diffuse rgb,
    specular rgb) for one direction pair, RGB."""
    out = np.zeros(3, np.float32)
    lib().svfo_pseudo_volume_rgb(np.ascontiguousarray(params_rgb, np.float32),
                                 np.ascontiguousarray(lights_parabolic, np.float32), view, light, bounces, samples,
                                 seed, out)
    return out


def lsq_fit_ms(lum, lights_parabolic, init7, bounces, max_steps=1024):
    """The reference LM on the pseudo-volume model (svbrdffit -m bounces)."""
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    out = np.zeros(7, np.float32)
    st = LsqStats()
    rmse = lib().svfo_lsq_fit_ms(np.ascontiguousarray(lum, np.float32), lp, lp.shape[0], bounces, max_steps,
                                 np.ascontiguousarray(init7, np.float32), out, C.byref(st))
    return out, float(rmse), st


def lsq_fit(lum, lights_parabolic, init7, fresnel=1.0, max_steps=1024):
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    out = np.zeros(7, np.float32)
    st = LsqStats()
    rmse = lib().svfo_lsq_fit(np.ascontiguousarray(lum, np.float32), lp, lp.shape[0], fresnel, max_steps,
                              np.ascontiguousarray(init7, np.float32), out, C.byref(st))
    return out, float(rmse), st


def lum_slice(rgb):
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    lum = np.zeros(rgb.shape[0], np.float32)
    avg = np.zeros(3, np.float32)
    lib().svfo_lum_slice(rgb, rgb.shape[0], lum, avg)
    return lum, avg


class MeshData:
    """Direction table plus the interpolation mesh (triangles, boundary edges)."""

    def __init__(self, lights_parabolic, triangles, edges, edge_angles):
        self.lights_parabolic = np.ascontiguousarray(lights_parabolic, np.float32)
        self.triangles = np.ascontiguousarray(triangles, np.uint32)
        self.edges = np.ascontiguousarray(edges, np.uint32)
        self.edge_angles = np.ascontiguousarray(edge_angles, np.float32)

    def cstruct(self) -> Mesh:
        return Mesh(self.lights_parabolic.ctypes.data, self.lights_parabolic.shape[0],
                    self.triangles.ctypes.data, self.triangles.shape[0],
                    self.edges.ctypes.data, self.edge_angles.ctypes.data, self.edges.shape[0])

    def save(self, path):
        np.savez(path, lights_parabolic=self.lights_parabolic, triangles=self.triangles,
                 edges=self.edges, edge_angles=self.edge_angles)

    @staticmethod
    def load(path) -> "MeshData":
        z = np.load(path)
        return MeshData(z["lights_parabolic"], z["triangles"], z["edges"], z["edge_angles"])


def ndf_texture(mesh: MeshData, lum) -> np.ndarray:
    ndf = np.zeros(64 * 64, np.float32)
    m = mesh.cstruct()
    lib().svfo_ndf_texture(C.byref(m), np.ascontiguousarray(lum, np.float32), ndf)
    return ndf


def default_init_from_ndf(ndf):
    init = np.zeros(7, np.float32)
    info = InitInfo()
    lib().svfo_default_init_from_ndf(np.ascontiguousarray(ndf, np.float32), init, C.byref(info))
    return init, info


def euler_to_matrix(euler3):
    m = np.zeros(9, np.float32)
    q = np.zeros(4, np.float32)
    lib().svfo_euler_to_matrix(np.ascontiguousarray(euler3, np.float32), m.ctypes.data, q.ctypes.data)
    return m.reshape(3, 3), q  # m[c] is column c


def synth_truth(seed, mix, texel) -> Truth:
    t = Truth()
    lib().svfo_synth_truth(seed, mix, texel, C.byref(t))
    return t


def synth_render(seed, texel, truth: Truth, lights_parabolic, noise=0.01):
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    L = lp.shape[0]
    rgb = np.zeros((L * L, 3), np.float32)
    lib().svfo_synth_render(seed, texel, C.byref(truth), lp, L, noise, rgb)
    return rgb


def truth_lum_params(t: Truth) -> np.ndarray:
    """The 7 luminance-model parameters of a synthetic texel."""
    kd = np.array(t.kd[:], np.float32)
    ks = np.array(t.ks[:], np.float32)
    w = np.array([0.2126, 0.7152, 0.0722], np.float32)
    return np.array([t.sigma[0], t.sigma[1], float(ks @ w), float(kd @ w), *t.euler[:]], np.float32)


# ----------------------------------------------------------------------------
# DFMF writer (the layout LoadBTF parses, src/image/btf.cc:389-1000)
# ----------------------------------------------------------------------------


def write_dfmf(path, theta_phi, rgb_texels, width=None, height=1, data_size=4):
    """Writes texels [T][N][3] as a DFMF BTF whose SVD factors reproduce the
    samples exactly: per channel, U = samples^T ([N][K], K = T) and SxV = I.

    Texel t sits at file column t; LoadBTF flips rows (btf.cc:1000-1022), so with
    height 1 texel t is at (x = t, y = 0) after loading.
    """
    rgb_texels = np.asarray(rgb_texels, np.float32)
    T, N, _ = rgb_texels.shape
    L = theta_phi.shape[0]
    assert N == L * L
    width = width or T
    assert width * height == T
    dt = {2: np.float16, 4: np.float32, 8: np.float64}[data_size]
    with open(path, "wb") as f:
        f.write(b"!")
        f.write(b"DFMF")
        f.write(b"08FC")
        # BTFCommonHeader (btf.hh:48-57): Size, Version, 3x80 chars, PPMM, RGB
        hdr = struct.pack("<II", 264, 1) + b"\0" * 240 + struct.pack("<f3f", 0.0, 1.0, 1.0, 1.0)
        assert len(hdr) == 264
        f.write(hdr)
        f.write(struct.pack("<I", L))
        tp = np.ascontiguousarray(theta_phi, np.float32)
        for v in range(L):
            f.write(tp[v].tobytes())
            f.write(struct.pack("<I", L))
            f.write(tp.tobytes())
        f.write(struct.pack("<II", width, height))
        f.write(struct.pack("<II", T, 0))                 # num_components, ColorModel
        f.write(struct.pack("<3f", 0.0, 0.0, 0.0))        # ColorMean
        f.write(np.eye(3, dtype=np.float32).tobytes())    # ColorTransform
        eye = np.eye(T, dtype=dt)
        for c in range(3):
            f.write(struct.pack("<B", data_size))
            f.write(struct.pack("<III", T, N, T))
            f.write(np.ones(T, dt).tobytes())             # scalars
            u = np.ascontiguousarray(rgb_texels[:, :, c].T.astype(dt))   # [N][K]
            f.write(u.tobytes())
            f.write(eye.tobytes())                         # SxV [cols][K]


def btf_file_bytes(theta_phi, width, height, planes, fmt="DFMF", data_size=4, color_model=0, drr=0,
                   version=1, cosine_flag=0, xml=b"", channel_names=None, rotations=None, ext_version=1,
                   heightmap=None, tail=b""):
    """The bytes of a factored BTF file in the layout LoadBTF parses (src/image/btf.cc:389-1028).

    planes: DFMF -- three (U [L*L][K_c], SxV [W*H][K_c]) pairs, one per channel;
            FMF0 / FMF1 -- one (U [L*L*3][K], SxV [W*H][K]) pair, U rows interleaved by channel.
    SxV rows are file columns: LoadBTF flips rows, so texel (x, y) reads column (H-1-y)*W + x.
    version (BTFCommonHeader::Version) > 1 adds the cosine flag, > 2 an XML string, > 3 the
    channel names; rotations (an [n][3][3] array) sets the 'R' marker; FMF1's ext_version >= 1
    stores drr, >= 2 the height map ([h][w] uint16).  tail: bytes appended after the data.
    """
    import io

    dt = {2: np.float16, 4: np.float32, 8: np.float64}[data_size]
    tp = np.ascontiguousarray(theta_phi, np.float32)
    L = tp.shape[0]
    f = io.BytesIO()
    f.write(b"!" + fmt.encode())
    f.write({"DFMF": b"08FC", "FMF1": b"2FCE", "FMF0": b"6FC"}[fmt])
    if rotations is not None:
        f.write(b"R")
    names = channel_names if channel_names is not None else [b"R", b"G", b"B"]
    extra = b""
    if version > 1:
        extra += struct.pack("<I", cosine_flag)
    if version > 2:
        extra += struct.pack("<I", len(xml)) + xml
    if version > 3:
        extra += struct.pack("<I", len(names)) + b"".join(struct.pack("<I", len(n)) + n for n in names)
    size = 264 + len(extra)
    f.write(struct.pack("<II", size, version) + b"\0" * 240 + struct.pack("<f3f", 0.0, 1.0, 1.0, 1.0))
    f.write(extra)
    f.write(struct.pack("<I", L))
    for v in range(L):
        f.write(tp[v].tobytes())
        f.write(struct.pack("<I", L))
        f.write(tp.tobytes())
    f.write(struct.pack("<II", width, height))
    if rotations is not None:
        rot = np.ascontiguousarray(rotations, np.float32)
        f.write(struct.pack("<I", rot.shape[0]) + rot.tobytes())
    if fmt == "DFMF":
        f.write(struct.pack("<II", planes[0][0].shape[1], color_model))
        f.write(struct.pack("<3f", 0.0, 0.0, 0.0))
        f.write(np.eye(3, dtype=np.float32).tobytes())
        for U, S in planes:
            K = U.shape[1]
            f.write(struct.pack("<B", data_size))
            f.write(struct.pack("<III", K, U.shape[0], S.shape[0]))
            f.write(np.ones(K, dt).tobytes())
            f.write(np.ascontiguousarray(U, dt).tobytes())
            f.write(np.ascontiguousarray(S, dt).tobytes())
    else:
        if fmt == "FMF1":
            f.write(struct.pack("<B", ext_version))
            if ext_version >= 1:
                f.write(struct.pack("<I", drr))
            if ext_version >= 2:
                hm = np.zeros((0, 0), np.uint16) if heightmap is None else np.ascontiguousarray(heightmap, np.uint16)
                f.write(struct.pack("<II", hm.shape[1], hm.shape[0]) + hm.tobytes())
        U, S = planes
        K = U.shape[1]
        f.write(struct.pack("<I", K) + struct.pack("<B", data_size) + struct.pack("<I", K))
        f.write(struct.pack("<II", U.shape[0], S.shape[0]))
        f.write(np.ones(K, dt).tobytes())
        f.write(np.ascontiguousarray(U, dt).tobytes())
        f.write(np.ascontiguousarray(S, dt).tobytes())
    f.write(tail)
    return f.getvalue()


class BtfPlanes(C.Structure):
    _fields_ = [("data_size", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("light_count", C.c_uint32), ("color_model", C.c_uint32), ("drr", C.c_uint32),
                ("u", C.c_void_p * 3), ("sxv", C.c_void_p * 3), ("k", C.c_uint32 * 3),
                ("u_row", C.c_uint64 * 3), ("sxv_row", C.c_uint64 * 3)]


def btf_decode(planes, fmt, width, height, light_count, data_size, color_model=0, drr=0, first=0, count=None):
    """The oracle's BTFFetchSpectrum over texels [first, first + count): [count][L*L][3] float32."""
    dt = {2: np.float16, 4: np.float32, 8: np.float64}[data_size]
    p = BtfPlanes()
    p.data_size, p.width, p.height, p.light_count = data_size, width, height, light_count
    p.color_model, p.drr = color_model, drr
    keep = []
    if fmt == "DFMF":
        for c, (U, S) in enumerate(planes):
            U = np.ascontiguousarray(U, dt)
            S = np.ascontiguousarray(S, dt)
            keep += [U, S]
            p.u[c], p.sxv[c], p.k[c] = U.ctypes.data, S.ctypes.data, U.shape[1]
            p.u_row[c], p.sxv_row[c] = U.shape[1], S.shape[1]
    else:
        U = np.ascontiguousarray(planes[0], dt)
        S = np.ascontiguousarray(planes[1], dt)
        keep += [U, S]
        K = U.shape[1]
        for c in range(3):
            p.u[c] = U.ctypes.data + c * K * data_size
            p.sxv[c], p.k[c] = S.ctypes.data, K
            p.u_row[c], p.sxv_row[c] = 3 * K, K
    count = width * height - first if count is None else count
    out = np.zeros((count, light_count * light_count, 3), np.float32)
    lib().svfo_btf_decode(C.byref(p), first, count, out.ctypes.data)
    return out


# ----------------------------------------------------------------------------
# the reference build
# ----------------------------------------------------------------------------

_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


# The reference pipeline with the drop-in LeastSquaresFitSGGX (svf_shim.cc on
# libsvf.so) in place of its CPU one: the same harness entry points.
REF_SVF_SO = os.path.join(HERE, "_ref", "libtempest_ref_svf.so")
_ref_svf = None


def ref_svf_available() -> bool:
    return os.path.exists(REF_SVF_SO)


def ref_svf():
    global _ref_svf
    if _ref_svf is None:
        _ref_svf = _bind_harness(C.CDLL(REF_SVF_SO))
    return _ref_svf


def ref():
    global _ref
    if _ref is None:
        _ref = _bind_harness(C.CDLL(REF_SO))
    return _ref


def _bind_harness(L):
    if True:
        L.ref_btf_load.argtypes = [C.c_char_p]
        L.ref_btf_load.restype = C.c_void_p
        L.ref_btf_free.argtypes = [C.c_void_p]
        L.ref_btf_info.argtypes = [C.c_void_p, _u32p]
        L.ref_btf_geometry.argtypes = [C.c_void_p, _f32p, _u32p, _u32p, _f32p]
        L.ref_btf_fetch.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _f32p]
        L.ref_btf_lum_slice.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _f32p, _f32p]
        L.ref_brdf_eval.argtypes = [_f32p, C.c_uint32, C.c_float, _f64p, _f32p]
        L.ref_lsq.argtypes = [_f32p, C.c_uint32, _f32p, C.c_float, C.c_uint32, _f32p, _f32p,
                              C.POINTER(C.c_float), _u32p]
        L.ref_fit_texel.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, _f32p, _f32p, _f32p,
                                    C.POINTER(C.c_float), _u32p, C.c_void_p, C.c_void_p]
        L.ref_fit_texel.restype = C.c_int
        L.ref_fit_texel_opts.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_uint32,
                                         C.c_uint32, _f32p, _f32p, _f32p, C.POINTER(C.c_float), _u32p]
        L.ref_fit_texel_opts.restype = C.c_int
        L.ref_time_fit_texels.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_float, C.c_void_p]
        L.ref_time_fit_texels.restype = C.c_double
        L.ref_exr_save.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32, _f32p]
        L.ref_exr_save.restype = C.c_int
        L.ref_exr_load.argtypes = [C.c_char_p, _u32p, C.c_void_p]
        L.ref_exr_load.restype = C.c_int
        L.ref_error_texel.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _f32p, _f32p, _f32p, _f32p, C.c_uint32,
                                      C.c_uint32, _f32p, _f32p]
        L.ref_lsq_opts.argtypes = [_f32p, C.c_uint32, _f32p, C.c_float, C.c_uint32, C.c_uint32, _f32p, _f32p,
                                   C.POINTER(C.c_float), _u32p]
        L.ref_brdf_eval_ms.argtypes = [_f32p, C.c_uint32, C.c_uint32, C.c_float, _f64p, _f32p]
        L.ref_lsq_ms.argtypes = [_f32p, C.c_uint32, _f32p, C.c_float, C.c_uint32, C.c_uint32, _f32p, _f32p,
                                 C.POINTER(C.c_float), _u32p]
        if hasattr(L, "ref_downsample"):   # (not in the seam library)
            L.ref_downsample.argtypes = [_f32p, C.c_uint32, _f32p, C.c_uint32, _f32p, _f32p]
    return L


LSF_OPTON_DIFFUSE = 1 << 1
LSF_OPTION_DISABLE_DIRECTION_FITTING = 1 << 2
LSF_OPTION_FIT_TOP = 1 << 4


class RefBTF:
    """A BTF loaded by the reference's LoadBTF."""

    def __init__(self, path, lib=None):
        """lib: the harness library that loads and fits it (default: the reference's own)."""
        self.lib = lib or ref()
        self.handle = self.lib.ref_btf_load(path.encode())
        if not self.handle:
            raise RuntimeError(f"LoadBTF failed on {path}")
        dims = np.zeros(5, np.uint32)
        self.lib.ref_btf_info(self.handle, dims)
        self.width, self.height, self.light_count, self.tri_count, self.edge_count = map(int, dims)

    @staticmethod
    def from_texels(theta_phi, rgb_texels, data_size=4, lib=None) -> "RefBTF":
        fd, path = tempfile.mkstemp(suffix=".btf")
        os.close(fd)
        try:
            write_dfmf(path, theta_phi, rgb_texels, data_size=data_size)
            return RefBTF(path, lib)
        finally:
            os.unlink(path)

    def mesh(self) -> MeshData:
        L = self.light_count
        lp = np.zeros((L, 2), np.float32)
        tri = np.zeros((self.tri_count, 3), np.uint32)
        e = np.zeros((self.edge_count, 3), np.uint32)
        ea = np.zeros((self.edge_count, 2), np.float32)
        self.lib.ref_btf_geometry(self.handle, lp, tri, e, ea)
        return MeshData(lp, tri, e, ea)

    def lum_slice(self, x, y=0):
        N = self.light_count ** 2
        lum = np.zeros(N, np.float32)
        avg = np.zeros(3, np.float32)
        self.lib.ref_btf_lum_slice(self.handle, x, y, lum, avg)
        return lum, avg

    def fit_texel(self, x, y=0, fresnel=1.0, want_ndf=False):
        init7 = np.zeros(7, np.float32)
        fit7 = np.zeros(7, np.float32)
        maps = np.zeros(12, np.float32)
        rmse = C.c_float()
        st = np.zeros(2, np.uint32)
        ndf = np.zeros(64 * 64, np.float32) if want_ndf else None
        rc = self.lib.ref_fit_texel(self.handle, x, y, fresnel, init7, fit7, maps, C.byref(rmse), st,
                                 ndf.ctypes.data if want_ndf else None, None)
        if rc != 0:
            raise RuntimeError("reference pipeline did not reach LeastSquaresFitSGGX")
        return dict(init=init7, fit=fit7, maps=maps, rmse=rmse.value, iterations=int(st[0]),
                    effective=int(st[1]), ndf=ndf)

    def fit_texel_opts(self, x, y=0, fresnel=1.0, flags=LSF_OPTON_DIFFUSE, downsample=0xFFFFFFFF,
                       bounces=0xFFFFFFFF):
        """The pipeline's fit of texel (x, y) with the given LeastSquaresFitOptions."""
        init7, fit7, maps = np.zeros(7, np.float32), np.zeros(7, np.float32), np.zeros(12, np.float32)
        rmse = C.c_float()
        st = np.zeros(2, np.uint32)
        rc = self.lib.ref_fit_texel_opts(self.handle, x, y, fresnel, flags, downsample, bounces, init7, fit7, maps,
                                         C.byref(rmse), st)
        if rc != 0:
            raise RuntimeError("reference pipeline did not reach LeastSquaresFitSGGX")
        return dict(init=init7, fit=fit7, maps=maps, rmse=rmse.value, iterations=int(st[0]), effective=int(st[1]))

    def time_fit(self, first, count, workers, pool_threads, fresnel=1.0):
        rm = np.zeros(count, np.float32)
        secs = self.lib.ref_time_fit_texels(self.handle, first, count, workers, pool_threads, fresnel,
                                         rm.ctypes.data)
        return secs, rm

    def __del__(self):
        try:
            if self.handle:
                self.lib.ref_btf_free(self.handle)
        except Exception:
            pass


def ref_lsq(lum, lights_parabolic, init7, fresnel=1.0, flags=LSF_OPTON_DIFFUSE):
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    out = np.zeros(7, np.float32)
    rmse = C.c_float()
    st = np.zeros(2, np.uint32)
    ref().ref_lsq(lp, lp.shape[0], np.ascontiguousarray(lum, np.float32), fresnel, flags,
                  np.ascontiguousarray(init7, np.float32), out, C.byref(rmse), st)
    return out, rmse.value, int(st[0]), int(st[1])


def ref_lsq_opts(lum, lights_parabolic, init7, fresnel=1.0, flags=LSF_OPTON_DIFFUSE, downsample=0xFFFFFFFF):
    """LeastSquaresFitSGGX with the given LeastSquaresFitOptions flags and DownSampleLightView."""
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    out = np.zeros(7, np.float32)
    rmse = C.c_float()
    st = np.zeros(2, np.uint32)
    ref().ref_lsq_opts(lp, lp.shape[0], np.ascontiguousarray(lum, np.float32), fresnel, flags, downsample,
                       np.ascontiguousarray(init7, np.float32), out, C.byref(rmse), st)
    return out, rmse.value, int(st[0]), int(st[1])


def ref_downsample(lum, lights_parabolic, n):
    """DownsampleLightView: the kept directions and the n x n slice."""
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    dirs = np.zeros((n, 2), np.float32)
    sl = np.zeros(n * n, np.float32)
    ref().ref_downsample(lp, lp.shape[0], np.ascontiguousarray(lum, np.float32), n, dirs, sl)
    return dirs, sl


def ref_lsq_ms(lum, lights_parabolic, init7, bounces, fresnel=1.0, flags=LSF_OPTON_DIFFUSE):
    """LeastSquaresFitSGGX with MultiScatteringBounceCount = bounces (the pseudo-volume model)."""
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    out = np.zeros(7, np.float32)
    rmse = C.c_float()
    st = np.zeros(2, np.uint32)
    ref().ref_lsq_ms(lp, lp.shape[0], np.ascontiguousarray(lum, np.float32), fresnel, flags, bounces,
                     np.ascontiguousarray(init7, np.float32), out, C.byref(rmse), st)
    return out, rmse.value, int(st[0]), int(st[1])


def ref_brdf_all_ms(params7, lights_parabolic, bounces, fresnel=1.0):
    """The reference's BRDFEvaluator with BounceCount = bounces over all pairs."""
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    L = lp.shape[0]
    out = np.zeros(L * L, np.float32)
    ref().ref_brdf_eval_ms(lp, L, bounces, fresnel, np.ascontiguousarray(params7, np.float64), out)
    return out


def ref_brdf_all(params7, lights_parabolic, fresnel=1.0):
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    L = lp.shape[0]
    out = np.zeros(L * L, np.float32)
    ref().ref_brdf_eval(lp, L, fresnel, np.ascontiguousarray(params7, np.float64), out)
    return out
