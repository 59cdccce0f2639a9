"""B200 SVBRDF fitting (Lambert + anisotropic SGGX, Levenberg-Marquardt) over libsvf.so.

Python mirror of the library's C ABI (``include/svf.h``), named after the
reference interfaces it replaces:

* :func:`lsq_fit_sggx` -- ``LeastSquaresFitSGGX``
  (tools/svbrdf-fitting/svbrdf-fitting.hh:126-127), one texel;
* :func:`lsq_fit_batch` -- the same fit for many texels in one launch;
* :func:`fit_texels` -- the svbrdffit texel loop (``PusherThread::execute``,
  svbrdf-fitting.cc:86-121, over ``SVBRDFFitPipeline::cache/fit``).

The library is the in-tree ``libsvf.so`` (``python -m tempestrenderer_b200.build``).
Nothing here computes on the CPU: when the library or a B200 is missing, the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsvf.so")

SVF_OK, SVF_EINVAL, SVF_ENOMEM, SVF_ECUDA, SVF_ETIMEOUT, SVF_EPARTIAL, SVF_ENODEV = range(7)
SVF_TEXEL_NONFINITE, SVF_TEXEL_MAX_ITER, SVF_TEXEL_TIMEOUT = 1, 2, 4
SVF_LSQ_DIFFUSE = 1 << 1
SVF_LSQ_RGB = 1 << 8
SVF_LSQ_STEP_PER_PARAMETER = 1 << 9
SVF_LSQ_DISABLE_DIRECTION_FITTING = 1 << 2
SVF_LSQ_FIT_TOP = 1 << 4
SVF_LSQ_MULTI_SCATTERING = 1 << 10
SVF_SAMPLES_F32, SVF_SAMPLES_F16 = 0, 1
SVF_INIT_DEFAULT, SVF_INIT_GIVEN, SVF_INIT_MLP = 0, 1, 2
SVF_ERROR_PAIRWISE, SVF_ERROR_MAX_VIEW = 0, 1
SVF_MLP_FEATURES_PAIRS_RGB, SVF_MLP_FEATURES_BINS = 0, 1
SVF_NOALLOC_MAX_SLAB_FLOATS = 1 << 19   # include/svf.h

# every entry point include/svf.h declares
EXPORTS = ("svf_abi_version", "svf_status_string", "svf_last_error", "svf_lsq_options_default", "svf_create",
           "svf_destroy", "svf_directions_ring81", "svf_directions_fibonacci", "svf_layout_triangulate",
           "svf_lsq_fit_sggx", "svf_lsq_fit_batch", "svf_lsq_fit_batch_noalloc", "svf_fit_texels", "svf_fit_btfs",
           "svf_synth_btf", "svf_mlp_train_options_default", "svf_mlp_train", "svf_mlp_predict", "svf_mlp_step",
           "svf_mlp_save", "svf_mlp_load", "svf_mlp_destroy", "svf_btf_probe", "svf_btf_load", "svf_btf_load_file",
           "svf_btf_get_info", "svf_btf_decode", "svf_fit_btf", "svf_btf_destroy", "svf_error_maps", "svf_exr_write",
           "svf_exr_read", "svf_maps_write_exr", "svf_params_from_maps", "svf_refit_neighborhood",
           "svf_render_btf", "svf_downsample_light_view", "svf_render_btf_ms")


class SvfError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"svf status {status}: {message}")
        self.status = status


class LsqOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_uint32), ("fresnel", C.c_float), ("flags", C.c_uint32),
                ("mse_target", C.c_double), ("break_on_small_step", C.c_double), ("restarts", C.c_uint32),
                ("downsample_light_view", C.c_uint32), ("multi_scattering_bounces", C.c_uint32)]


class TexelStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("effective", C.c_uint32), ("jacobians", C.c_uint32),
                ("residuals", C.c_uint32), ("status", C.c_uint32)]


STATS_DTYPE = np.dtype([("iterations", np.uint32), ("effective", np.uint32), ("jacobians", np.uint32),
                        ("residuals", np.uint32), ("status", np.uint32)])


class LayoutDesc(C.Structure):
    _fields_ = [("lights_parabolic", C.c_void_p), ("light_count", C.c_uint32), ("triangles", C.c_void_p),
                ("triangle_count", C.c_uint32), ("edges", C.c_void_p), ("edge_angles", C.c_void_p),
                ("edge_count", C.c_uint32)]


class BtfView(C.Structure):
    _fields_ = [("samples", C.c_void_p), ("sample_type", C.c_uint32), ("width", C.c_uint32),
                ("height", C.c_uint32), ("layout", C.POINTER(LayoutDesc))]


class FitOptions(C.Structure):
    _fields_ = [("lsq", LsqOptions), ("init_mode", C.c_uint32), ("init_params", C.c_void_p), ("mlp", C.c_void_p),
                ("initial_damping", C.c_float), ("mlp_fallback", C.c_float)]


class BtfInfo(C.Structure):
    _fields_ = [("format", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("light_count", C.c_uint32),
                ("data_size", C.c_uint32), ("color_model", C.c_uint32), ("dynamic_range_reduction", C.c_uint32),
                ("cosine_flag", C.c_uint32), ("version", C.c_uint32), ("components", C.c_uint32 * 3)]


class SvbrdfMaps(C.Structure):
    _fields_ = [("diffuse", C.c_void_p), ("specular", C.c_void_p), ("sigma", C.c_void_p),
                ("sigma_channels", C.c_uint32), ("basis", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32)]


class MlpTrainOptions(C.Structure):
    _fields_ = [("texels", C.c_uint32), ("seed", C.c_uint32), ("mix", C.c_uint32), ("epochs", C.c_uint32),
                ("batch", C.c_uint32), ("lr", C.c_float), ("max_iterations", C.c_uint32),
                ("features", C.c_uint32)]


class Maps(C.Structure):
    _fields_ = [("diffuse", C.c_void_p), ("specular", C.c_void_p), ("sigma", C.c_void_p), ("basis", C.c_void_p),
                ("rmse", C.c_void_p), ("params", C.c_void_p), ("init", C.c_void_p), ("stats", C.c_void_p),
                ("ndf", C.c_void_p)]


class RunStats(C.Structure):
    _fields_ = [("texels", C.c_uint64), ("iterations", C.c_uint64), ("jacobians", C.c_uint64),
                ("residuals", C.c_uint64), ("failed_texels", C.c_uint64), ("ms_total", C.c_double),
                ("ms_luminance", C.c_double), ("ms_init", C.c_double), ("ms_fit", C.c_double),
                ("ms_copy", C.c_double), ("lm_threads", C.c_uint32), ("lm_slots", C.c_uint32),
                ("ms_ndf", C.c_double), ("graph", C.c_uint32), ("fallback_texels", C.c_uint32),
                ("ndf_tiles", C.c_uint32), ("ndf_tiles_total", C.c_uint32)]


_lib = None


def load() -> C.CDLL:
    """Loads the in-tree libsvf.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run `python -m tempestrenderer_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float
        L.svf_abi_version.restype = u32
        L.svf_status_string.argtypes = [C.c_int]
        L.svf_status_string.restype = C.c_char_p
        L.svf_last_error.restype = C.c_char_p
        L.svf_lsq_options_default.argtypes = [C.POINTER(LsqOptions)]
        L.svf_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.svf_destroy.argtypes = [vp]
        L.svf_directions_ring81.argtypes = [vp]
        L.svf_directions_ring81.restype = u32
        L.svf_directions_fibonacci.argtypes = [u32, vp]
        L.svf_directions_fibonacci.restype = u32
        L.svf_downsample_light_view.argtypes = [u32, u32, vp]
        L.svf_downsample_light_view.restype = u32
        L.svf_layout_triangulate.argtypes = [vp, u32, vp, vp, vp, C.POINTER(u32)]
        L.svf_layout_triangulate.restype = u32
        L.svf_lsq_fit_sggx.argtypes = [vp, vp, u32, vp, C.POINTER(LsqOptions), vp, vp, vp, C.POINTER(TexelStats)]
        L.svf_lsq_fit_batch.argtypes = [vp, vp, u32, vp, u64, u32, C.POINTER(LsqOptions), vp, vp, vp, vp]
        L.svf_lsq_fit_batch_noalloc.argtypes = [vp, u32, vp, u64, u32, C.POINTER(LsqOptions), vp, vp, vp, vp, vp]
        L.svf_fit_texels.argtypes = [vp, C.POINTER(BtfView), C.POINTER(FitOptions), C.POINTER(Maps),
                                     C.POINTER(RunStats)]
        L.svf_synth_btf.argtypes = [vp, u32, u32, vp, u32, u64, u64, u32, f32, vp, vp]
        L.svf_fit_btfs.argtypes = [vp, C.POINTER(BtfView), u32, C.POINTER(FitOptions), C.POINTER(Maps),
                                   C.POINTER(RunStats), C.POINTER(RunStats)]
        L.svf_mlp_train_options_default.argtypes = [C.POINTER(MlpTrainOptions)]
        L.svf_mlp_train_options_default.restype = None
        L.svf_mlp_train.argtypes = [vp, vp, u32, C.POINTER(MlpTrainOptions), C.POINTER(vp), C.POINTER(f32)]
        L.svf_mlp_predict.argtypes = [vp, vp, vp, u32, u32, vp, vp]
        L.svf_mlp_step.argtypes = [vp, vp, vp, vp, u32, f32, u32, C.POINTER(f32)]
        L.svf_mlp_save.argtypes = [vp, vp, C.POINTER(C.c_size_t)]
        L.svf_mlp_load.argtypes = [vp, vp, C.c_size_t, C.POINTER(vp)]
        L.svf_mlp_destroy.argtypes = [vp]
        L.svf_mlp_destroy.restype = None
        L.svf_btf_probe.argtypes = [vp, C.c_size_t, C.POINTER(BtfInfo), vp]
        L.svf_btf_load.argtypes = [vp, vp, C.c_size_t, C.POINTER(vp)]
        L.svf_btf_load_file.argtypes = [vp, C.c_char_p, C.POINTER(vp)]
        L.svf_btf_get_info.argtypes = [vp, C.POINTER(BtfInfo), vp]
        L.svf_btf_decode.argtypes = [vp, vp, u64, u64, u32, vp]
        L.svf_fit_btf.argtypes = [vp, vp, vp, C.POINTER(FitOptions), C.POINTER(Maps), C.POINTER(RunStats)]
        L.svf_btf_destroy.argtypes = [vp]
        L.svf_btf_destroy.restype = None
        L.svf_error_maps.argtypes = [vp, vp, C.POINTER(SvbrdfMaps), u32, u32, u32, u32, vp, vp]
        L.svf_exr_write.argtypes = [C.c_char_p, u32, u32, u32, vp]
        L.svf_exr_read.argtypes = [C.c_char_p, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), vp, C.c_size_t]
        L.svf_maps_write_exr.argtypes = [C.c_char_p, u32, u32, C.POINTER(Maps)]
        L.svf_params_from_maps.argtypes = [C.POINTER(SvbrdfMaps), vp, vp]
        L.svf_render_btf.argtypes = [vp, vp, u32, C.POINTER(SvbrdfMaps), f32, u32, vp]
        L.svf_render_btf_ms.argtypes = [vp, vp, u32, C.POINTER(SvbrdfMaps), u32, u32, u32, u32, vp]
        L.svf_refit_neighborhood.argtypes = [vp, C.POINTER(BtfView), C.POINTER(LsqOptions), vp, vp, C.POINTER(Maps),
                                             C.POINTER(RunStats)]
        for name in ("svf_create", "svf_lsq_fit_sggx", "svf_lsq_fit_batch", "svf_lsq_fit_batch_noalloc",
                     "svf_fit_texels", "svf_fit_btfs", "svf_synth_btf", "svf_mlp_train", "svf_mlp_predict",
                     "svf_mlp_step", "svf_mlp_save", "svf_mlp_load", "svf_btf_probe", "svf_btf_load",
                     "svf_btf_load_file", "svf_btf_get_info", "svf_btf_decode", "svf_fit_btf", "svf_error_maps",
                     "svf_exr_write", "svf_exr_read", "svf_maps_write_exr", "svf_params_from_maps",
                     "svf_refit_neighborhood", "svf_render_btf", "svf_render_btf_ms"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _check(status: int):
    if status != SVF_OK:
        raise SvfError(status, load().svf_last_error().decode())


def options(max_iterations: int = 1024, fresnel: float = 1.0, restarts: int | None = None,
            rgb: bool = False, step_per_parameter: bool = True, diffuse: bool = True,
            fit_direction: bool = True, downsample: int = 0, fit_top: bool = False,
            multi_scattering: int | None = None) -> LsqOptions:
    """LM options; rgb selects the 11-parameter RGB fit (svf_fit_texels / svf_fit_btfs);
    step_per_parameter=False restores the reference's whole-vector small-step test;
    diffuse=False the specular-only fit, fit_direction=False holds the Euler angles,
    downsample=n fits n of the directions, multi_scattering=bounces the pseudo-volume
    model (svf_lsq_fit_sggx / svf_lsq_fit_batch)."""
    o = LsqOptions()
    load().svf_lsq_options_default(C.byref(o))
    o.max_iterations = max_iterations
    o.fresnel = fresnel
    o.downsample_light_view = downsample
    if multi_scattering is not None:
        o.flags |= SVF_LSQ_MULTI_SCATTERING
        o.multi_scattering_bounces = multi_scattering
    if not diffuse:
        o.flags &= ~SVF_LSQ_DIFFUSE
    if not fit_direction:
        o.flags |= SVF_LSQ_DISABLE_DIRECTION_FITTING
    if fit_top:
        o.flags |= SVF_LSQ_FIT_TOP
    if rgb:
        o.flags |= SVF_LSQ_RGB
    if not step_per_parameter:
        o.flags &= ~SVF_LSQ_STEP_PER_PARAMETER
    if restarts is not None:
        o.restarts = restarts
    return o


def _ptr(a) -> int:
    """Address of a numpy array (host) or a torch tensor (device or host)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return a.data_ptr()  # torch.Tensor


def directions_ring81() -> np.ndarray:
    lp = np.zeros((81, 2), np.float32)
    n = load().svf_directions_ring81(lp.ctypes.data)
    assert n == 81
    return lp


def downsample_light_view(light_count: int, n: int) -> np.ndarray:
    """The direction indices DownsampleLightView keeps (svf_downsample_light_view)."""
    idx = np.zeros(max(n, 1), np.uint32)[:n]
    if n < 2 or load().svf_downsample_light_view(light_count, n, idx.ctypes.data) != n:
        raise SvfError(SVF_EINVAL, f"no draw of {n} of {light_count} directions")
    return idx


def directions_fibonacci(count: int) -> np.ndarray:
    lp = np.zeros((count, 2), np.float32)
    load().svf_directions_fibonacci(count, lp.ctypes.data)
    return lp


def triangulate(lights_parabolic: np.ndarray):
    lp = np.ascontiguousarray(lights_parabolic, np.float32)
    L = lp.shape[0]
    tri = np.zeros((2 * L, 3), np.uint32)
    e = np.zeros((L, 3), np.uint32)
    ea = np.zeros((L, 2), np.float32)
    ne = C.c_uint32()
    nt = load().svf_layout_triangulate(lp.ctypes.data, L, tri.ctypes.data, e.ctypes.data, ea.ctypes.data,
                                       C.byref(ne))
    if nt == 0:
        raise SvfError(SVF_EINVAL, "triangulation failed")
    return tri[:nt].copy(), e[:ne.value].copy(), ea[:ne.value].copy()


class Layout:
    """A direction layout and, optionally, its interpolation mesh (BTF::LightIndices/Edges)."""

    def __init__(self, lights_parabolic, triangles=None, edges=None, edge_angles=None):
        self.lights_parabolic = np.ascontiguousarray(lights_parabolic, np.float32)
        self.triangles = None if triangles is None else np.ascontiguousarray(triangles, np.uint32)
        self.edges = None if edges is None else np.ascontiguousarray(edges, np.uint32)
        self.edge_angles = None if edge_angles is None else np.ascontiguousarray(edge_angles, np.float32)
        d = LayoutDesc()
        d.lights_parabolic = self.lights_parabolic.ctypes.data
        d.light_count = self.lights_parabolic.shape[0]
        if self.triangles is not None:
            d.triangles = self.triangles.ctypes.data
            d.triangle_count = self.triangles.shape[0]
            d.edges = self.edges.ctypes.data
            d.edge_angles = self.edge_angles.ctypes.data
            d.edge_count = self.edges.shape[0]
        self.desc = d

    @property
    def light_count(self) -> int:
        return self.lights_parabolic.shape[0]


class Context:
    """A device context (svf_create / svf_destroy)."""

    def __init__(self, device: int = 0):
        self._lib = load()
        h = C.c_void_p()
        _check(self._lib.svf_create(device, C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self._lib.svf_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # LeastSquaresFitSGGX -------------------------------------------------------
    def lsq_fit_sggx(self, lights_parabolic, lum, init7, opts: LsqOptions | None = None):
        lp = np.ascontiguousarray(lights_parabolic, np.float32)
        lum = np.ascontiguousarray(lum, np.float32)
        init = np.ascontiguousarray(init7, np.float32)
        out = np.zeros(7, np.float32)
        rmse = np.zeros(1, np.float32)
        st = TexelStats()
        o = opts or options()
        _check(self._lib.svf_lsq_fit_sggx(self.handle, lp.ctypes.data, lp.shape[0], lum.ctypes.data, C.byref(o),
                                          init.ctypes.data, out.ctypes.data, rmse.ctypes.data, C.byref(st)))
        return out, float(rmse[0]), st

    def lsq_fit_batch(self, lights_parabolic, lum, init, opts: LsqOptions | None = None, out=None, rmse=None,
                      stats=None):
        """lum: [T][stride] (numpy or torch, host or device); init: [T][7]."""
        lp = np.ascontiguousarray(lights_parabolic, np.float32)
        T = int(lum.shape[0])
        stride = int(lum.shape[1])
        if out is None:
            out = np.zeros((T, 7), np.float32)
        if rmse is None:
            rmse = np.zeros(T, np.float32)
        if stats is None:
            stats = np.zeros(T, STATS_DTYPE)
        o = opts or options()
        _check(self._lib.svf_lsq_fit_batch(self.handle, lp.ctypes.data, lp.shape[0], _ptr(lum), stride, T,
                                           C.byref(o), _ptr(init), _ptr(out), _ptr(rmse), _ptr(stats)))
        return out, rmse, stats

    # svbrdffit texel loop -------------------------------------------------------
    def fit_texels(self, layout: Layout, samples, width: int, height: int, sample_type=SVF_SAMPLES_F32,
                   opts: LsqOptions | None = None, init=None, want=("diffuse", "specular", "sigma", "basis", "rmse",
                                                                    "params", "init", "stats"), out=None,
                   check=True, mlp: "Mlp | None" = None, damping: float = 0.0, fallback: float = 0.0):
        """samples: [T][L*L][3] (numpy or torch, host or device).  init: given initial parameters; mlp: a
        learned initial guess (SVF_INIT_MLP); neither: the default guess.  damping: LM's initial damping as a
        multiple of the reference's rule (0: automatic).  Returns (maps dict, RunStats)."""
        T = width * height
        v = BtfView()
        v.samples = _ptr(samples)
        v.sample_type = sample_type
        v.width, v.height = width, height
        v.layout = C.pointer(layout.desc)
        fo = FitOptions()
        fo.lsq = opts or options()
        fo.init_mode = SVF_INIT_DEFAULT if init is None else SVF_INIT_GIVEN
        fo.init_params = _ptr(init) if init is not None else None
        if mlp is not None:
            fo.init_mode, fo.mlp = SVF_INIT_MLP, mlp.handle
        fo.initial_damping = damping
        fo.mlp_fallback = fallback
        kout = 12 if fo.lsq.flags & SVF_LSQ_RGB else 7
        shapes = {"diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4), "rmse": (T,),
                  "params": (T, kout), "init": (T, kout), "ndf": (T, 64 * 64)}
        res = dict(out or {})
        for k in want:
            if k in res:
                continue
            res[k] = np.zeros(T, STATS_DTYPE) if k == "stats" else np.zeros(shapes[k], np.float32)
        m = Maps()
        for k in ("diffuse", "specular", "sigma", "basis", "rmse", "params", "init", "stats", "ndf"):
            setattr(m, k, _ptr(res[k]) if k in res else None)
        rs = RunStats()
        st = self._lib.svf_fit_texels(self.handle, C.byref(v), C.byref(fo), C.byref(m), C.byref(rs))
        if check:
            _check(st)
        return res, rs

    def fit_btfs(self, btfs, opts: LsqOptions | None = None, want=("diffuse", "specular", "sigma", "basis", "rmse",
                                                                  "params", "init", "stats"), check=True):
        """btfs: list of dicts {layout, samples, width, height[, sample_type][, init][, mlp]}.  All texels go through
        shared LM launches (svf_fit_btfs).  Returns ([maps dict per BTF], [RunStats per BTF], RunStats total)."""
        n = len(btfs)
        views = (BtfView * n)()
        fos = (FitOptions * n)()
        ms = (Maps * n)()
        keep, results = [], []
        for i, b in enumerate(btfs):
            T = b["width"] * b["height"]
            views[i].samples = _ptr(b["samples"])
            views[i].sample_type = b.get("sample_type", SVF_SAMPLES_F32)
            views[i].width, views[i].height = b["width"], b["height"]
            views[i].layout = C.pointer(b["layout"].desc)
            fos[i].lsq = opts or options()
            init = b.get("init")
            fos[i].init_mode = SVF_INIT_DEFAULT if init is None else SVF_INIT_GIVEN
            if b.get("mlp") is not None:
                fos[i].init_mode, fos[i].mlp = SVF_INIT_MLP, b["mlp"].handle
            fos[i].initial_damping = b.get("damping", 0.0)
            if init is not None:
                init = np.ascontiguousarray(init, np.float32)
                keep.append(init)
                fos[i].init_params = init.ctypes.data
            kout = 12 if fos[i].lsq.flags & SVF_LSQ_RGB else 7
            shapes = {"diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4), "rmse": (T,),
                      "params": (T, kout), "init": (T, kout), "ndf": (T, 64 * 64)}
            res = {k: (np.zeros(T, STATS_DTYPE) if k == "stats" else np.zeros(shapes[k], np.float32)) for k in want}
            for k in ("diffuse", "specular", "sigma", "basis", "rmse", "params", "init", "stats", "ndf"):
                setattr(ms[i], k, _ptr(res[k]) if k in res else None)
            results.append(res)
        runs = (RunStats * n)()
        total = RunStats()
        st = self._lib.svf_fit_btfs(self.handle, views, n, fos, ms, runs, C.byref(total))
        if check:
            _check(st)
        return results, list(runs), total

    def refit_neighborhood(self, layout: Layout, samples, width: int, height: int, params, rmse,
                           sample_type=SVF_SAMPLES_F32, opts: LsqOptions | None = None,
                           want=("params", "rmse", "diffuse", "specular", "sigma", "basis")):
        """svbrdffit -j as one GPU pass (svf_refit_neighborhood).  Returns (maps dict, RunStats)."""
        T = width * height
        v = BtfView()
        v.samples = _ptr(samples)
        v.sample_type = sample_type
        v.width, v.height = width, height
        v.layout = C.pointer(layout.desc)
        # numpy arrays or torch tensors (host or device)
        p = params if hasattr(params, "data_ptr") else np.ascontiguousarray(params, np.float32)
        r = rmse if hasattr(rmse, "data_ptr") else np.ascontiguousarray(rmse, np.float32)
        shapes = {"diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4), "rmse": (T,),
                  "params": (T, 7)}
        res = {k: np.zeros(shapes[k], np.float32) for k in want}
        m = Maps()
        for k in ("diffuse", "specular", "sigma", "basis", "rmse", "params"):
            setattr(m, k, _ptr(res[k]) if k in res else None)
        rs = RunStats()
        _check(self._lib.svf_refit_neighborhood(self.handle, C.byref(v), C.byref(opts or options()), _ptr(p),
                                                _ptr(r), C.byref(m), C.byref(rs)))
        return res, rs

    def render_btf(self, lights_parabolic, diffuse, specular, sigma, basis, fresnel: float = 1.0,
                   sample_type=SVF_SAMPLES_F32, out=None):
        """Samples [texels][L*L][3] of SVBRDF maps ([texels][3|3|2or3|4]) -- svf_render_btf."""
        lp = np.ascontiguousarray(lights_parabolic, np.float32)
        d, sp, sg, b = (np.ascontiguousarray(m, np.float32).reshape(-1, m.shape[-1]) for m in
                        (np.asarray(diffuse), np.asarray(specular), np.asarray(sigma), np.asarray(basis)))
        T, L = d.shape[0], lp.shape[0]
        m = SvbrdfMaps(d.ctypes.data, sp.ctypes.data, sg.ctypes.data, sg.shape[1], b.ctypes.data, T, 1)
        if out is None:
            out = np.zeros((T, L * L, 3), np.float16 if sample_type == SVF_SAMPLES_F16 else np.float32)
        _check(self._lib.svf_render_btf(self.handle, lp.ctypes.data, L, C.byref(m), fresnel, sample_type, _ptr(out)))
        return out

    def render_btf_ms(self, lights_parabolic, diffuse, specular, sigma, basis, bounces: int, samples: int = 256,
                      seed: int = 0, sample_type=SVF_SAMPLES_F32, out=None):
        """Samples [texels][L*L][3] of SVBRDF maps with the pseudo-volume multi-scattering
        BRDF -- svf_render_btf_ms."""
        lp = np.ascontiguousarray(lights_parabolic, np.float32)
        d, sp, sg, b = (np.ascontiguousarray(m, np.float32).reshape(-1, m.shape[-1]) for m in
                        (np.asarray(diffuse), np.asarray(specular), np.asarray(sigma), np.asarray(basis)))
        T, L = d.shape[0], lp.shape[0]
        m = SvbrdfMaps(d.ctypes.data, sp.ctypes.data, sg.ctypes.data, sg.shape[1], b.ctypes.data, T, 1)
        if out is None:
            out = np.zeros((T, L * L, 3), np.float16 if sample_type == SVF_SAMPLES_F16 else np.float32)
        _check(self._lib.svf_render_btf_ms(self.handle, lp.ctypes.data, L, C.byref(m), bounces, samples, seed,
                                           sample_type, _ptr(out)))
        return out

    def synth_btf(self, seed: int, mix: int, lights_parabolic, first: int, count: int, samples,
                  sample_type=SVF_SAMPLES_F32, noise: float = 0.01, truth=None):
        lp = np.ascontiguousarray(lights_parabolic, np.float32)
        _check(self._lib.svf_synth_btf(self.handle, seed, mix, lp.ctypes.data, lp.shape[0], first, count,
                                       sample_type, noise, _ptr(samples), _ptr(truth)))


def mlp_train_options(**kw) -> MlpTrainOptions:
    o = MlpTrainOptions()
    load().svf_mlp_train_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Mlp:
    """A learned initial guess (svf_mlp_*).  Create with Mlp.train or Mlp.load."""

    def __init__(self, ctx: Context, handle):
        self._lib, self.ctx, self.handle = load(), ctx, handle

    @classmethod
    def train(cls, ctx: Context, lights_parabolic, opts: MlpTrainOptions | None = None):
        """Returns (model, final epoch's loss on the normalised targets)."""
        lp = np.ascontiguousarray(lights_parabolic, np.float32)
        h, loss = C.c_void_p(), C.c_float()
        _check(load().svf_mlp_train(ctx.handle, lp.ctypes.data, lp.shape[0], C.byref(opts or mlp_train_options()),
                                    C.byref(h), C.byref(loss)))
        return cls(ctx, h), float(loss.value)

    @classmethod
    def load(cls, ctx: Context, blob: bytes):
        h = C.c_void_p()
        buf = C.create_string_buffer(bytes(blob), len(blob))
        _check(load().svf_mlp_load(ctx.handle, buf, len(blob), C.byref(h)))
        return cls(ctx, h)

    def save(self) -> bytes:
        n = C.c_size_t(0)
        _check(self._lib.svf_mlp_save(self.handle, None, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(self._lib.svf_mlp_save(self.handle, buf, C.byref(n)))
        return buf.raw[:n.value]

    def predict(self, samples, texels: int, sample_type=SVF_SAMPLES_F32, features=False):
        """Initial parameters [texels][7] (and the normalised inputs [texels][96] with features=True)."""
        p = np.zeros((texels, 7), np.float32)
        f = np.zeros((texels, 96), np.float32) if features else None
        _check(self._lib.svf_mlp_predict(self.ctx.handle, self.handle, _ptr(samples), sample_type, texels,
                                         p.ctypes.data, f.ctypes.data if features else None))
        return (p, f) if features else p

    def step(self, features, targets, lr: float, sgd: bool = False) -> float:
        """One optimiser step; returns the MSE before it."""
        x = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(targets, np.float32)
        loss = C.c_float()
        _check(self._lib.svf_mlp_step(self.ctx.handle, self.handle, x.ctypes.data, y.ctypes.data, x.shape[0], lr,
                                      int(sgd), C.byref(loss)))
        return float(loss.value)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.svf_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


def btf_probe(data: bytes):
    """Parses a DFMF / FMF file image on the host: (BtfInfo, lights_parabolic [L][2])."""
    info = BtfInfo()
    lp = np.zeros((160, 2), np.float32)
    buf = C.create_string_buffer(bytes(data), len(data))
    _check(load().svf_btf_probe(buf, len(data), C.byref(info), lp.ctypes.data))
    return info, lp[:info.light_count].copy()


class Btf:
    """A factored BTF file loaded onto a context's device (svf_btf_*)."""

    def __init__(self, ctx: Context, data: bytes | None = None, path: str | None = None):
        self._lib, self.ctx = load(), ctx
        h = C.c_void_p()
        if path is not None:
            _check(self._lib.svf_btf_load_file(ctx.handle, path.encode(), C.byref(h)))
        else:
            buf = C.create_string_buffer(bytes(data), len(data))
            _check(self._lib.svf_btf_load(ctx.handle, buf, len(data), C.byref(h)))
        self.handle = h
        self.info = BtfInfo()
        lp = np.zeros((160, 2), np.float32)
        _check(self._lib.svf_btf_get_info(h, C.byref(self.info), lp.ctypes.data))
        self.lights_parabolic = lp[:self.info.light_count].copy()

    @property
    def texels(self) -> int:
        return self.info.width * self.info.height

    def decode(self, first: int = 0, count: int | None = None, sample_type=SVF_SAMPLES_F32, out=None):
        """RGB samples [count][L*L][3] (numpy on the host unless `out` is given)."""
        count = self.texels - first if count is None else count
        N = self.info.light_count ** 2
        if out is None:
            out = np.zeros((count, N, 3), np.float16 if sample_type == SVF_SAMPLES_F16 else np.float32)
        _check(self._lib.svf_btf_decode(self.ctx.handle, self.handle, first, count, sample_type, _ptr(out)))
        return out

    def fit(self, layout: "Layout | None" = None, opts: LsqOptions | None = None, init=None, mlp=None,
            want=("diffuse", "specular", "sigma", "basis", "rmse", "params", "init", "stats"), check=True):
        """svf_fit_btf: layout (optional) supplies the default guess's interpolation mesh."""
        T = self.texels
        fo = FitOptions()
        fo.lsq = opts or options()
        fo.init_mode = SVF_INIT_DEFAULT if init is None else SVF_INIT_GIVEN
        fo.init_params = _ptr(init) if init is not None else None
        if mlp is not None:
            fo.init_mode, fo.mlp = SVF_INIT_MLP, mlp.handle
        kout = 12 if fo.lsq.flags & SVF_LSQ_RGB else 7
        shapes = {"diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4), "rmse": (T,),
                  "params": (T, kout), "init": (T, kout), "ndf": (T, 64 * 64)}
        res = {k: (np.zeros(T, STATS_DTYPE) if k == "stats" else np.zeros(shapes[k], np.float32)) for k in want}
        m = Maps()
        for k in ("diffuse", "specular", "sigma", "basis", "rmse", "params", "init", "stats", "ndf"):
            setattr(m, k, _ptr(res[k]) if k in res else None)
        rs = RunStats()
        mesh = C.pointer(layout.desc) if layout is not None else None
        st = self._lib.svf_fit_btf(self.ctx.handle, self.handle, mesh, C.byref(fo), C.byref(m), C.byref(rs))
        if check:
            _check(st)
        return res, rs

    def error_maps(self, diffuse, specular, sigma, basis, x0: int = 0, y0: int = 0, method=SVF_ERROR_PAIRWISE,
                   color: bool = False):
        """svbrdf-error-tool: maps [h][w][3|3|2or3|4] -> (rmse, psnr) [h][w] ([h][w][3] with color)."""
        d, sp, sg, b = (np.ascontiguousarray(m, np.float32) for m in (diffuse, specular, sigma, basis))
        h, w = d.shape[:2]
        m = SvbrdfMaps(d.ctypes.data, sp.ctypes.data, sg.ctypes.data, sg.shape[2], b.ctypes.data, w, h)
        shape = (h, w, 3) if color else (h, w)
        rmse, psnr = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
        _check(self._lib.svf_error_maps(self.ctx.handle, self.handle, C.byref(m), x0, y0, method, int(color),
                                        rmse.ctypes.data, psnr.ctypes.data))
        return rmse, psnr

    def close(self):
        if getattr(self, "handle", None):
            self._lib.svf_btf_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


def exr_write(path: str, image) -> None:
    """An [h][w] or [h][w][c] float image (c = 1..4) as svbrdffit saves its maps."""
    img = np.ascontiguousarray(image, np.float32)
    if img.ndim == 2:
        img = img[:, :, None]
    _check(load().svf_exr_write(path.encode(), img.shape[1], img.shape[0], img.shape[2], img.ctypes.data))


def exr_read(path: str) -> np.ndarray:
    """[h][w][c] float32 from an uncompressed OpenEXR file (LoadEXRImage's layout)."""
    w, h, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    _check(load().svf_exr_read(path.encode(), C.byref(w), C.byref(h), C.byref(c), None, 0))
    out = np.zeros((h.value, w.value, c.value), np.float32)
    _check(load().svf_exr_read(path.encode(), C.byref(w), C.byref(h), C.byref(c), out.ctypes.data, out.size))
    return out


def maps_write_exr(prefix: str, width: int, height: int, maps: dict) -> None:
    """svbrdffit's <prefix>_albedo/_specular/_sggx_scale/_sggx_basis/_rmse.exr from host maps."""
    m = Maps()
    keep = {}
    for k in ("diffuse", "specular", "sigma", "basis", "rmse"):
        if k in maps:
            keep[k] = np.ascontiguousarray(maps[k], np.float32)
            setattr(m, k, keep[k].ctypes.data)
    _check(load().svf_maps_write_exr(prefix.encode(), width, height, C.byref(m)))


def params_from_maps(diffuse, specular, sigma, basis):
    """svbrdffit -r: the 7 fit parameters of saved maps (and the colour they carry)."""
    d, sp, sg, b = (np.ascontiguousarray(m, np.float32) for m in (diffuse, specular, sigma, basis))
    T = d.shape[0] * (d.shape[1] if d.ndim == 3 else 1)
    sc = sg.shape[-1]
    m = SvbrdfMaps(d.ctypes.data, sp.ctypes.data, sg.ctypes.data, sc, b.ctypes.data, T, 1)
    p = np.zeros((T, 7), np.float32)
    colour = np.zeros((T, 3), np.float32)
    _check(load().svf_params_from_maps(C.byref(m), p.ctypes.data, colour.ctypes.data))
    return p, colour
