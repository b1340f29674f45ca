"""gpv -- Python host interface of the B200 subset-correlation library.

Mirrors the reference package's Python classes for this path
(geopyv_dev/__init__.py:299-385 ``Subset``, python/src/py_image.rs:41-64
``Image``, python/src/py_mask.rs:89-154 ``Mask``) over the C ABI of
``include/gpv.h``.  All arithmetic runs in the CUDA library; this module only
marshals arguments.
"""
from __future__ import annotations

import ctypes as ct
import os
import threading

# Up to 32 hardware work queues instead of the driver's default 8, so that
# the streams of concurrent contexts (server workers, high-priority streams)
# do not share in-order queues, where a high-priority kernel would wait for a
# low-priority one ahead of it.  The driver reads it when CUDA initialises in
# the process, so it applies when this package is imported before any CUDA
# use; an explicit setting is kept.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import numpy as np

from . import _lib
from ._lib import (DESC_DTYPE, RESULT_DTYPE, PREC_FP64, PREC_MIXED, SOLVE_ETA, STATUS, GpvError, SolveParams,
                   check, lib, ptr)

__all__ = ["Context", "Image", "Mask", "Subset", "Mesh", "mesh_drive", "SubsetSequence", "Sequence", "Server", "solve_batch", "autotune", "make_desc", "DESC_DTYPE", "RESULT_DTYPE",
           "GpvError", "PREC_MIXED", "PREC_FP64", "STATUS", "version"]


def version() -> str:
    return lib().gpv_version().decode()


class Context:
    """One CUDA device, one stream and the solve workspace (gpv_context)."""

    def __init__(self, device: int = 0, high_priority: bool = False, per_subset_blocks: bool = False):
        """high_priority: streams at the device's greatest priority;
        per_subset_blocks: host-batch solves launch one block per subset
        instead of a persistent grid (gpv_context_create_ex)."""
        h = ct.c_void_p()
        flags = (_lib.CONTEXT_HIGH_PRIORITY if high_priority else 0) | \
            (_lib.CONTEXT_PER_SUBSET_BLOCKS if per_subset_blocks else 0)
        check(lib().gpv_context_create_ex(device, flags, ct.byref(h)), "gpv_context_create_ex")
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return lib().gpv_context_stream(self._h) or 0

    def tuning(self):
        """Tuned launch dimensions per radius class r <= 20, 21-40, > 40: a dict
        per class (threads per block, tiled-kernel template layout, run length,
        subsets per block, window staging; None where untuned)."""
        from ._lib import Tuning
        t = (Tuning * 3)()
        check(lib().gpv_context_tuning_get(self._h, t), "gpv_context_tuning_get")
        names = {-1: None, 0: "compact", 1: "rows", 2: "tiles"}
        return [{"threads": t[c].threads or None, "layout": names.get(t[c].layout), "run_length": t[c].run_length or None,
                 "subsets_per_block": t[c].subsets_per_block or None, "staging": t[c].staging or None}
                for c in range(3)]

    def reserve(self, n_subsets: int, max_radius: int, max_iterations: int = 50) -> None:
        check(lib().gpv_context_reserve(self._h, n_subsets, max_radius, max_iterations), "gpv_context_reserve")

    def close(self) -> None:
        if self._h:
            lib().gpv_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = {}
_default_lock = threading.Lock()


def default_context(device: int = 0) -> Context:
    with _default_lock:
        if device not in _default:
            _default[device] = Context(device)
        return _default[device]


class Image:
    """Device-resident bi-quintic B-spline coefficients of a greyscale image.

    ``Image(image_gs=array, border=20)`` as python/src/py_image.rs:42-64 (the
    coefficients are computed on the GPU: Image::from_array -> get_c,
    src/image.rs:83-86, :252-327).  ``keep_f64`` keeps an FP64 copy of the
    coefficients for the FP64 solver; ``grain`` keeps the rigid-texture grain
    maps (GrainMaps, src/texture.rs:31-143), rebuilt with every update.

    ``Image(image_rgb=array)`` takes decoded 8-bit colour pixels (h, w, 3) in
    RGB order and applies Image::from_file's pre-processing on the device
    (grey level, 5 x 5 Gaussian blur, rounding: src/image.rs:450-534) before
    the prefilter.  ``Image(filepath=...)`` decodes the file with OpenCV when
    it is installed and then does the same; lossless formats decode to the
    same pixels as the reference's decoder, lossy ones (JPEG) may differ by a
    grey level where the two decoders' inverse DCTs round differently.
    """

    def __init__(self, filepath=None, image_gs=None, border: int = 20, keep_f64: bool = False, ctx: Context | None = None,
                 image_rgb=None, grain: bool = False):
        given = [v is not None for v in (filepath, image_gs, image_rgb)]
        if sum(given) > 1:
            raise ValueError("supply exactly one of `filepath`, `image_gs` or `image_rgb`")
        if not any(given):
            raise ValueError("one of `filepath`, `image_gs` or `image_rgb` is required")
        if filepath is not None:
            try:
                import cv2
            except ImportError as e:  # pragma: no cover - depends on the installation
                raise NotImplementedError("decoding image files needs OpenCV; pass image_gs or image_rgb") from e
            bgr = cv2.imread(str(filepath), cv2.IMREAD_COLOR)
            if bgr is None:
                raise RuntimeError(f"image load error: cannot read {filepath}")
            image_rgb = np.ascontiguousarray(bgr[:, :, ::-1])
        self.ctx = ctx or default_context()
        self.border = border
        h = ct.c_void_p()
        flags = (_lib.IMAGE_KEEP_F64 if keep_f64 else 0) | (_lib.IMAGE_GRAIN if grain else 0)
        if image_rgb is not None:
            rgb = np.ascontiguousarray(image_rgb, dtype=np.uint8)
            if rgb.ndim != 3 or rgb.shape[2] != 3:
                raise ValueError("image_rgb must be (h, w, 3) uint8")
            self.shape = rgb.shape[:2]
            self.dtype = np.dtype(np.uint8)
            check(lib().gpv_image_create_rgb8(self.ctx.handle, ptr(rgb), rgb.shape[0], rgb.shape[1], border, flags,
                                              ct.byref(h)), "gpv_image_create_rgb8")
        else:
            arr = np.asarray(image_gs)
            if arr.ndim != 2:
                raise ValueError("image_gs must be 2-D")
            if arr.dtype not in _lib.DTYPES:
                arr = arr.astype(np.float64)
            arr = np.ascontiguousarray(arr)
            self.shape = arr.shape
            self.dtype = arr.dtype
            check(lib().gpv_image_create(self.ctx.handle, ptr(arr), _lib.DTYPES[arr.dtype], arr.shape[0], arr.shape[1],
                                         border, flags, ct.byref(h)), "gpv_image_create")
        self._h = h
        self.keep_f64 = keep_f64

    @property
    def image_gs(self) -> np.ndarray:
        """The greyscale pixels of an image built from colour pixels (float64, as the reference's image_gs)."""
        out = np.empty(self.shape, np.uint8)
        check(lib().gpv_image_grey(self._h, ptr(out)), "gpv_image_grey")
        return out.astype(np.float64)

    def build_grain(self) -> None:
        """Build (once) and keep the rigid-texture grain maps of this image
        (gpv_image_build_grain); a solve with texture="rigid" calls it on the
        reference image."""
        check(lib().gpv_image_build_grain(self._h), "gpv_image_build_grain")

    def grain(self, maps: bool = False) -> dict:
        """The grain statistics: correlation length, s2, smoothing correction,
        whether the image has measurable speckle, and (maps=True) the
        (3, h, w) FP32 maps fxx, fyy, fxy."""
        out = (ct.c_double * 3)()
        built = ct.c_int32()
        m = np.empty((3,) + tuple(self.shape), np.float32) if maps else None
        check(lib().gpv_image_grain(self._h, out, ct.byref(built), ptr(m)), "gpv_image_grain")
        r = dict(correlation_length=out[0], s2=out[1], corr=out[2], built=bool(built.value))
        if maps:
            r["maps"] = m
        return r

    def grain_sample(self, xy) -> np.ndarray:
        """(n, 3) fxx, fyy, fxy of the grain maps at points (x = column, y = row),
        sampled on the device as the solves sample them."""
        xy = np.ascontiguousarray(np.atleast_2d(xy), dtype=np.float64)
        out = np.empty((xy.shape[0], 3))
        check(lib().gpv_image_grain_sample(self._h, ptr(xy), xy.shape[0], ptr(out)), "gpv_image_grain_sample")
        return out

    def update_rgb(self, image_rgb) -> None:
        """Ingest and prefilter new colour pixels of the same shape in place."""
        rgb = np.ascontiguousarray(image_rgb, dtype=np.uint8)
        if rgb.shape != (*self.shape, 3):
            raise ValueError(f"shape {rgb.shape} != {(*self.shape, 3)}")
        check(lib().gpv_image_update_rgb8(self._h, ptr(rgb)), "gpv_image_update_rgb8")

    @property
    def handle(self):
        return self._h

    def update(self, image_gs) -> None:
        """Re-prefilter new pixels of the same shape into this image in place
        (gpv_image_update; a sequence's next frame, src/sequence.rs:914)."""
        arr = np.ascontiguousarray(image_gs)
        if arr.shape != tuple(self.shape):
            raise ValueError(f"shape {arr.shape} != {tuple(self.shape)}")
        if arr.dtype not in _lib.DTYPES:
            arr = np.ascontiguousarray(arr, dtype=np.float64)
        check(lib().gpv_image_update(self._h, ptr(arr), _lib.DTYPES[arr.dtype]), "gpv_image_update")

    def coef(self, f64: bool = False) -> np.ndarray:
        """Coefficient array C, shape (h + 2 border, w + 2 border) (src/image.rs:48-51)."""
        shp = (self.shape[0] + 2 * self.border, self.shape[1] + 2 * self.border)
        if f64:
            out = np.empty(shp, np.float64)
            check(lib().gpv_image_coefficients_f64(self._h, ptr(out)), "gpv_image_coefficients_f64")
        else:
            out = np.empty(shp, np.float32)
            check(lib().gpv_image_coefficients_f32(self._h, ptr(out)), "gpv_image_coefficients_f32")
        return out

    def eval(self, xy, grad: bool = False, precision: int = PREC_MIXED):
        """Spline value (and gradient) at points (x = column, y = row): Image::eval / eval_grad."""
        xy = np.ascontiguousarray(np.atleast_2d(xy), dtype=np.float64)
        n = xy.shape[0]
        val = np.empty(n)
        g = np.empty((n, 2)) if grad else None
        check(lib().gpv_image_eval(self._h, ptr(xy), n, precision, ptr(val), ptr(g)), "gpv_image_eval")
        return (val, g) if grad else val

    def close(self):
        if getattr(self, "_h", None):
            lib().gpv_image_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mask:
    """Local (circular template) or global (binary image) mask.

    ``Mask("local", shape="circle", size=25)`` as python/src/py_mask.rs:89-110;
    ``Mask("global", binary=array)`` takes the binary mask image directly
    (the reference rasterises it from boundary polygons, which is outside this
    library).
    """

    def __init__(self, mask_type: str, shape: str | None = None, size: int = 25, binary=None, ctx: Context | None = None):
        self.mask_type = mask_type
        self._h = None
        if mask_type == "local":
            if shape is None:
                raise ValueError("shape is required for mask_type='local'")
            if shape != "circle":
                raise NotImplementedError(f"local mask shape '{shape}': only 'circle' is supported")
            if size <= 0:
                raise RuntimeError("invalid input: radius must be > 0")
            self.shape, self.size = shape, int(size)
        elif mask_type == "global":
            if binary is None:
                raise ValueError("binary is required for mask_type='global'")
            b = np.ascontiguousarray(binary, dtype=np.uint8)
            self.binary = b
            self.ctx = ctx or default_context()
            h = ct.c_void_p()
            check(lib().gpv_mask_create(self.ctx.handle, ptr(b), b.shape[0], b.shape[1], ct.byref(h)),
                  "gpv_mask_create")
            self._h = h
        else:
            raise ValueError(f"unknown mask_type '{mask_type}': expected 'local' or 'global'")

    @property
    def n_px(self) -> int:
        r = self.size
        y, x = np.mgrid[-r:r + 1, -r:r + 1]
        return int(np.count_nonzero(x * x + y * y <= r * r))

    @property
    def handle(self):
        return self._h

    def __del__(self):
        try:
            if self._h:
                lib().gpv_mask_destroy(self._h)
        except Exception:
            pass


def make_desc(coords, radius, order, p0=None) -> np.ndarray:
    """Structured gpv_subset_desc array from centres (n, 2), radii and orders."""
    coords = np.atleast_2d(np.asarray(coords, dtype=np.float64))
    n = coords.shape[0]
    d = np.zeros(n, DESC_DTYPE)
    d["coord"] = coords
    d["radius"] = np.broadcast_to(np.asarray(radius, dtype=np.int32), (n,))
    d["order"] = np.broadcast_to(np.asarray(order, dtype=np.int32), (n,))
    if p0 is not None:
        p0 = np.atleast_2d(np.asarray(p0, dtype=np.float64))
        d["p0"][:, :p0.shape[1]] = p0
    return d


def _params(max_norm, max_iterations, tolerance, eta, precision, mask, history_buf, method="icgn",
            texture="deformable"):
    if method not in ("icgn", "fagn"):
        raise ValueError(f"method must be 'icgn' or 'fagn', got {method!r}")
    if texture not in ("deformable", "rigid"):  # check_texture (python/src/py_mesh.rs:954-961)
        raise ValueError(f"texture must be 'deformable' or 'rigid', got {texture!r}")
    flags = (SOLVE_ETA if eta else 0) | (_lib.SOLVE_FAGN if method == "fagn" else 0) | \
        (_lib.SOLVE_RIGID_TEXTURE if texture == "rigid" else 0)
    return SolveParams(max_norm=max_norm, tolerance=tolerance, max_iterations=max_iterations,
                       flags=flags, precision=precision, reserved=0,
                       mask=(mask.handle if mask is not None else None),
                       history=(history_buf.ctypes.data if history_buf is not None else None))


def solve_batch(f_img: Image, g_img: Image, desc, max_norm=1e-5, max_iterations=50, tolerance=0.75, eta=False,
                precision=PREC_MIXED, global_mask: Mask | None = None, history=False, method="icgn",
                texture="deformable"):
    """Batched Subset::new + solve_icgn_result on the GPU; returns a RESULT_DTYPE array
    (and the (n, max_iterations, 3) history of (norm, zncc, znssd) when asked).
    texture="rigid" fits the rigid-texture template (its ``texture`` field
    says whether a subset did)."""
    desc = np.ascontiguousarray(desc, dtype=DESC_DTYPE)
    out = np.zeros(desc.size, RESULT_DTYPE)
    hist = np.zeros((desc.size, max(max_iterations, 1), 3)) if history else None
    prm = _params(max_norm, max_iterations, tolerance, eta, precision, global_mask, hist, method, texture)
    if texture == "rigid":
        f_img.build_grain()
    check(lib().gpv_solve_batch(f_img.ctx.handle, f_img.handle, g_img.handle, ptr(desc), desc.size,
                                ct.byref(prm), ptr(out)), "gpv_solve_batch")
    return (out, hist) if history else out


def autotune(f_img: Image, g_img: Image, desc, max_norm=1e-5, max_iterations=50, tolerance=0.75,
             sample_per_class=1024):
    """Pick the fastest launch shape per radius class on a sample of `desc`
    (gpv_autotune); returns threads per subset block for r <= 20, 21..40, > 40."""
    desc = np.ascontiguousarray(desc, dtype=DESC_DTYPE)
    prm = _params(max_norm, max_iterations, tolerance, False, PREC_MIXED, None, None)
    out = (ct.c_int32 * 3)()
    check(lib().gpv_autotune(f_img.ctx.handle, f_img.handle, g_img.handle, ptr(desc), desc.size, ct.byref(prm),
                             sample_per_class, out), "gpv_autotune")
    return list(out)


class Subset:
    """One subset, solved on the GPU (geopyv_dev/__init__.py:299-385,
    python/src/py_subset.rs:159-237).  Results are read back as attributes
    (``p``, ``c_zncc``, ``c_znssd``, ``iterations``, ``converged``,
    ``quality_ok``, ``eta_omitted``, ``history``)."""

    def __init__(self, coord, local_mask: Mask, f_img: Image, g_img: Image, subset_order: int = 1,
                 global_mask: Mask | None = None):
        if subset_order > 2 or subset_order < 0:
            raise ValueError(f"subset_order must be 0, 1, or 2, got {subset_order}")
        if not isinstance(local_mask, Mask) or local_mask.mask_type != "local":
            raise TypeError("local_mask must be a Mask")
        self.coord = [float(coord[0]), float(coord[1])]
        self.local_mask, self.global_mask = local_mask, global_mask
        self.f_img, self.g_img = f_img, g_img
        self.subset_order = subset_order
        self._result = None
        self._history = None
        self._precision = PREC_MIXED
        self.solved = False

    def solve(self, p_0=None, solver=None, max_norm=1e-3, max_iterations=50, tolerance=0.75, precision=PREC_MIXED,
              algorithm=None, texture="deformable"):
        """Subset.solve: ``algorithm`` (or ``solver``) "icgn" (default) or "fagn";
        ``texture`` "deformable" (default) or "rigid"."""
        method = algorithm or solver or "icgn"
        if method not in ("icgn", "fagn"):
            raise ValueError(f"algorithm must be 'icgn' or 'fagn', got {method!r}")
        self._solve(method, p_0, max_norm, max_iterations, tolerance, precision, texture)

    def solve_icgn(self, p_0=None, max_norm=1e-3, max_iterations=50, tolerance=0.75, precision=PREC_MIXED,
                   texture="deformable"):
        self._solve("icgn", p_0, max_norm, max_iterations, tolerance, precision, texture)

    def solve_fagn(self, p_0=None, max_norm=1e-3, max_iterations=50, tolerance=0.75, precision=PREC_MIXED):
        """Forward additive Gauss-Newton (Subset::solve_fagn, src/subset.rs:1011-1020, 1228-1334)."""
        self._solve("fagn", p_0, max_norm, max_iterations, tolerance, precision)

    def _solve(self, method, p_0, max_norm, max_iterations, tolerance, precision, texture="deformable"):
        m = {0: 2, 1: 6, 2: 12}[self.subset_order]
        p0 = np.zeros(m)
        if p_0 is not None:  # resized to the order's length (src/subset.rs:1134-1136)
            v = np.asarray(p_0, dtype=np.float64).ravel()[:m]
            p0[:v.size] = v
        d = make_desc([self.coord], self.local_mask.size, self.subset_order, p0[None, :])
        out, hist = solve_batch(self.f_img, self.g_img, d, max_norm=max_norm, max_iterations=max_iterations,
                                tolerance=tolerance, eta=True, precision=precision, global_mask=self.global_mask,
                                history=True, method=method, texture=texture)
        r = out[0]
        st = int(r["status"])
        if st in (1, 2):  # Subset::new errors (src/subset.rs:853-892) -> RuntimeError (python/src/lib.rs:18-38)
            raise RuntimeError("invalid input: " + ("effective mask coords is empty" if st == 1
                                                    else "reference subset is featureless (delta_f = 0)"))
        if st in (3, 4):  # the reference panics (src/subset.rs:471,520,595,1143)
            what = "FAGN Hessian singular" if method == "fagn" else "ICGN Hessian singular"
            raise RuntimeError(what if st == 3 else "W_delta singular")
        self._result = r
        self._precision = precision
        k = int(r["iterations"])
        self._history = [(i + 1, *hist[0, i]) for i in range(k)]
        self.solved = True
        self.method = method

    def _get(self, key):
        if self._result is None:
            raise RuntimeError("Subset has not been solved; call solve() first")
        return self._result[key]

    @property
    def p(self):
        m = {0: 2, 1: 6, 2: 12}[self.subset_order]
        return np.array(self._get("p")[:m])

    c_zncc = property(lambda s: float(s._get("c_zncc")))
    c_znssd = property(lambda s: float(s._get("c_znssd")))
    # SolveResult::texture: the template the solve fitted
    texture = property(lambda s: "rigid" if int(s._get("texture")) else "deformable")
    iterations = property(lambda s: int(s._get("iterations")))
    converged = property(lambda s: bool(s._get("converged")))
    quality_ok = property(lambda s: bool(s._get("quality_ok")))
    f_m = property(lambda s: float(s._get("f_m")))
    delta_f = property(lambda s: float(s._get("delta_f")))
    sssig = property(lambda s: float(s._get("sssig")))
    sigma_intensity = property(lambda s: float(s._get("sigma")))
    n_px = property(lambda s: int(s._get("n_px")))
    history = property(lambda s: s._history)

    @property
    def f_coords(self) -> np.ndarray:
        """(n, 2) subset pixel coordinates: the circle's offsets in its scan
        order (LocalMask::circle, src/masks.rs:69-109) about the centre, less
        the pixels the global mask removes (mask_update, :199-263)."""
        r = self.local_mask.size
        y, x = np.mgrid[-r:r + 1, -r:r + 1]
        keep = x * x + y * y <= r * r
        off = np.column_stack([x[keep], y[keep]]).astype(np.float64)
        if self.global_mask is not None:
            b = self.global_mask.binary
            X = int(self.coord[0]) + off[:, 0].astype(np.int64)
            Y = int(self.coord[1]) + off[:, 1].astype(np.int64)
            ok = (X >= 0) & (Y >= 0) & (X <= b.shape[1] - 2) & (Y <= b.shape[0] - 2)
            ok[ok] = b[Y[ok], X[ok]] != 0
            off = off[ok]
        return off + np.array(self.coord)

    def _f_eval(self):
        prec = PREC_FP64 if self.f_img.keep_f64 else PREC_MIXED
        return self.f_img.eval(self.f_coords, grad=True, precision=prec)

    f = property(lambda s: s._f_eval()[0], doc="reference subset values (Subset::f)")
    grad_f = property(lambda s: s._f_eval()[1], doc="reference subset gradients (n, 2)")

    def residual_map(self) -> np.ndarray:
        """Per-pixel zero-normalised residual zn(f) - zn(g) at the solved warp,
        against the rigid-texture template when the solve fitted it
        (Subset::residual_map, src/subset.rs:1350-1392); the images are
        evaluated on the device."""
        if self._result is None:
            raise RuntimeError("invalid input: residual_map: subset has not been solved")
        fc = self.f_coords
        prec = self._precision if (self._precision == PREC_MIXED or
                                   (self.f_img.keep_f64 and self.g_img.keep_f64)) else PREC_MIXED
        f = self.f_img.eval(fc, precision=prec)
        m = {0: 2, 1: 6, 2: 12}[self.subset_order]
        p = np.zeros(12)
        p[:m] = self._get("p")[:m]
        dx, dy = fc[:, 0] - self.coord[0], fc[:, 1] - self.coord[1]
        xw = fc[:, 0] + p[0] + p[2] * dx + p[4] * dy + 0.5 * p[6] * dx * dx + p[8] * dx * dy + 0.5 * p[10] * dy * dy
        yw = fc[:, 1] + p[1] + p[3] * dx + p[5] * dy + 0.5 * p[7] * dx * dx + p[9] * dx * dy + 0.5 * p[11] * dy * dy
        g = self.g_img.eval(np.column_stack([xw, yw]), precision=prec)
        t = f
        if self.texture == "rigid":  # grain_template (src/texture.rs:213-244), base = the subset mean
            h = self.f_img.grain_sample(fc)
            if m <= 7:
                ux, vx, uy, vy = p[2], p[3], p[4], p[5]
            else:
                ux, vx = p[2] + p[6] * dx + p[8] * dy, p[3] + p[7] * dx + p[9] * dy
                uy, vy = p[4] + p[8] * dx + p[10] * dy, p[5] + p[9] * dx + p[11] * dy
            e0 = ux + 0.5 * (ux * ux + vx * vx)
            e1 = vy + 0.5 * (uy * uy + vy * vy)
            e2 = 0.5 * (uy + vx) + 0.5 * (ux * uy + vx * vy)
            s2 = self.f_img.grain()["s2"]
            t = f + (-0.5 * s2 * (e0 * h[:, 0] + e1 * h[:, 1] + 2.0 * e2 * h[:, 2]) - (e0 + e1) * (f - f.mean()))
        tm, gm = t.mean(), g.mean()
        return (t - tm) / np.sqrt(np.sum((t - tm) ** 2)) - (g - gm) / np.sqrt(np.sum((g - gm) ** 2))

    @property
    def eta_omitted(self):
        r = self._result
        return (float(r["eta_u"]), float(r["eta_v"])) if r is not None and r["has_eta"] else None


from .mesh import Cancelled, Mesh, mesh_drive  # noqa: E402  (uses the classes above only through arguments)
from .server import Server, Ticket  # noqa: E402
from . import sequence  # noqa: E402
from .sequence import Sequence  # noqa: E402


class SubsetSequence:
    """Frame-to-frame tracking of a fixed set of subsets (gpv_sequence_*):
    the per-frame work of Sequence.solve (src/sequence.rs:624-968) with the
    reference image fixed, every frame's target re-prefiltered in place and
    each subset seeded from its own last converged solution on the device.
    From the second frame on, the frame's device work is one CUDA graph
    (``graph=False`` launches it eagerly instead)."""

    def __init__(self, f_img: Image, g_img: Image, desc, dtype, max_norm=1e-5, max_iterations=50, tolerance=0.75,
                 precision=PREC_MIXED, global_mask: Mask | None = None, graph: bool = True):
        desc = np.ascontiguousarray(desc, dtype=DESC_DTYPE)
        self.n = desc.size
        self.dtype = np.dtype(dtype)
        if self.dtype not in _lib.DTYPES:
            raise TypeError(f"unsupported pixel dtype {self.dtype}")
        self.shape = f_img.shape
        self._imgs = (f_img, g_img, global_mask)  # kept alive while the sequence exists
        prm = _params(max_norm, max_iterations, tolerance, False, precision, global_mask, None)
        h = ct.c_void_p()
        check(lib().gpv_sequence_create(f_img.ctx.handle, f_img.handle, g_img.handle, ptr(desc), self.n,
                                        ct.byref(prm), _lib.DTYPES[self.dtype], 0 if graph else 1, ct.byref(h)),
              "gpv_sequence_create")
        self._h = h

    def frame(self, px=None, device_ptr: int | None = None, download: bool = True):
        """Solve one frame from host pixels `px` (h x w of the sequence's
        dtype) or from device pixels at `device_ptr`; returns the results
        (RESULT_DTYPE) when `download`, else None (results stay on the device)."""
        out = np.zeros(self.n, RESULT_DTYPE) if download else None
        if device_ptr is not None:
            rc = lib().gpv_sequence_frame(self._h, ct.c_void_p(device_ptr), 1, ptr(out))
        else:
            a = np.ascontiguousarray(px, dtype=self.dtype)
            if a.shape != tuple(self.shape):
                raise ValueError(f"frame shape {a.shape} != {tuple(self.shape)}")
            rc = lib().gpv_sequence_frame(self._h, ptr(a), 0, ptr(out))
        check(rc, "gpv_sequence_frame")
        return out

    def results_device(self) -> int:
        """Device address of the last frame's results (valid until the next frame)."""
        return int(lib().gpv_sequence_results_device(self._h) or 0)

    @property
    def frames(self) -> int:
        return int(lib().gpv_sequence_frames(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().gpv_sequence_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
