"""The reference's plugin classes, B200-backed.

Names, setters, defaults and call order follow yorsh87/nicp (nicp/nicp/*.h);
storage is device-resident and every compute call goes through the C ABI of
libnicp_b200.so (include/nicp_gpu.h).  Typical use mirrors
nicp_simple_aligner.cpp:100-165:

    proj = PinholePointProjector(); proj.setCameraMatrix(K); proj.setImageSize(480, 640)
    stats = StatsCalculatorIntegralImage()
    pim, nim = PointInformationMatrixCalculator(), NormalInformationMatrixCalculator()
    conv = DepthImageConverterIntegralImage(proj, stats, pim, nim)
    ref, cur = Cloud(), Cloud()
    conv.compute(ref, depth0); conv.compute(cur, depth1)
    cf = CorrespondenceFinderProjective(); lin = Linearizer()
    aligner = AlignerProjective(proj, lin, cf)
    aligner.setReferenceCloud(ref); aligner.setCurrentCloud(cur); aligner.align()
    T = aligner.T()
"""
import ctypes as C
import math

import numpy as np

from . import _lib as L


# ------------------------------------------------------------------ context
class Context:
    """A device, a CUDA stream and the library workspace (nicp_ctx)."""

    _default = None

    def __init__(self, device=0, stream=None):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.nicp_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(h))
        if rc != L.NICP_OK:
            raise L.NicpError(rc, "cannot create a context on device %d (an sm_100 GPU is required)" % device)
        self.h = h

    @classmethod
    def default(cls):
        if cls._default is None:
            cls._default = Context()
        return cls._default

    def check(self, rc):
        L.check(rc, self.h)

    def synchronize(self):
        self.check(self.lib.nicp_ctx_synchronize(self.h))

    def stream(self):
        return self.lib.nicp_ctx_stream(self.h)

    def device_bytes(self):
        return self.lib.nicp_ctx_device_bytes(self.h)

    def kernel_launches(self):
        return self.lib.nicp_ctx_kernel_launches(self.h)

    def transfer_bytes(self):
        h, d = C.c_ulonglong(0), C.c_ulonglong(0)
        self.check(self.lib.nicp_ctx_transfer_bytes(self.h, C.byref(h), C.byref(d)))
        return h.value, d.value

    def set_profiling(self, on):
        self.check(self.lib.nicp_ctx_set_profiling(self.h, 1 if on else 0))

    def set_autotune(self, on):
        """Per resolution mix, pick the fastest launch shapes on first use."""
        self.check(self.lib.nicp_ctx_set_autotune(self.h, 1 if on else 0))

    def launch_shape(self):
        """(z-buffer points per thread, fused-kernel CTAs per SM (0 = all that
        fit), resolution mixes tuned) of the last alignment call."""
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        self.check(self.lib.nicp_ctx_launch_shape(self.h, C.byref(a), C.byref(b), C.byref(c), None, None))
        return a.value, b.value, c.value

    def stats_shape(self):
        """(threads per CTA, CTAs per SM) of the stats kernel in the last build."""
        a, b = C.c_int(0), C.c_int(0)
        self.check(self.lib.nicp_ctx_launch_shape(self.h, None, None, None, C.byref(a), C.byref(b)))
        return a.value, b.value

    def read_profile(self, kernel):
        ms = C.c_double(0)
        n = C.c_int(0)
        self.check(self.lib.nicp_ctx_read_profile(self.h, L.K[kernel] if isinstance(kernel, str) else kernel,
                                                  C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.nicp_ctx_destroy(self.h)
            self.h = None
            if Context._default is self:
                Context._default = None


# ------------------------------------------------------------------ data model
class Cloud:
    """A device-resident cloud (cloud.h:20-193): points, normals, curvature
    (Stats::curvature), point and normal information matrices."""

    def __init__(self, ctx=None):
        self.ctx = ctx or Context.default()
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.nicp_cloud_create(self.ctx.h, C.byref(h)))
        self.h = h
        self.has_stats = False

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                self.ctx.lib.nicp_cloud_destroy(self.h)
        except Exception:
            pass

    def size(self):
        n = C.c_int(0)
        self.ctx.check(self.ctx.lib.nicp_cloud_size(self.h, C.byref(n)))
        return n.value

    __len__ = size

    def normal_count(self):
        """Points with a normal (counted on the device by the build)."""
        n = C.c_int(0)
        self.ctx.check(self.ctx.lib.nicp_cloud_normal_count(self.h, C.byref(n)))
        return n.value

    def download(self, stats=False):
        n = self.size()
        p = np.zeros((n, 4), np.float32)
        nn = np.zeros((n, 4), np.float32)
        k = np.zeros(n, np.float32)
        op = np.zeros((n, 9), np.float32)
        on = np.zeros((n, 9), np.float32)
        ev = np.zeros((n, 3), np.float32) if stats else None
        U = np.zeros((n, 9), np.float32) if stats else None
        self.ctx.check(self.ctx.lib.nicp_cloud_download(self.h, L.fptr(p), L.fptr(nn), L.fptr(k), L.fptr(op),
                                                        L.fptr(on), L.fptr(ev), L.fptr(U)))
        out = dict(points=p, normals=nn, curvature=k, omega_p=op.reshape(n, 3, 3), omega_n=on.reshape(n, 3, 3))
        if stats:
            out["eigenvalues"] = ev
            out["eigenvectors"] = U.reshape(n, 3, 3)
        return out

    def stats(self):
        """Stats per point (keep_stats): dict of eigenvalues (n x 3),
        eigenvectors (n x 3 x 3, columns), mean (n x 3), n (window points)."""
        k = self.size()
        ev, U, m = np.zeros((k, 3), np.float32), np.zeros((k, 9), np.float32), np.zeros((k, 3), np.float32)
        cnt = np.zeros(k, np.int32)
        self.ctx.check(self.ctx.lib.nicp_cloud_download_stats(self.h, L.fptr(ev), L.fptr(U), L.fptr(m), L.iptr(cnt)))
        return dict(eigenvalues=ev, eigenvectors=U.reshape(k, 3, 3), mean=m, n=cnt)

    def gaussians(self):
        """Cloud::gaussians() (cloud.h:107): (means n x 3, covariances n x 3 x 3);
        the cloud must have been built with keepGaussians."""
        n = self.size()
        m = np.zeros((n, 3), np.float32)
        c = np.zeros((n, 9), np.float32)
        self.ctx.check(self.ctx.lib.nicp_cloud_download_gaussians(self.h, L.fptr(m), L.fptr(c)))
        return m, c.reshape(n, 3, 3)

    def points(self):
        return self.download()["points"]

    def normals(self):
        return self.download()["normals"]

    def save(self, filename, T=None, step=1, binary=True):
        """Cloud::save (cloud.cpp:20-25,100-150): the reference's .nicp file."""
        self.ctx.check(self.ctx.lib.nicp_cloud_save(self.h, str(filename).encode(), L.fptr(L.f16(T)), int(step),
                                                    1 if binary else 0))
        return True

    def load(self, filename, params=None):
        """Cloud::load (cloud.cpp:13-18,42-98): returns the file's pose T; the
        information matrices are recomputed with `params` (CloudParams,
        default the calculators' defaults)."""
        T = np.zeros(16, np.float32)
        n = C.c_int(0)
        self.ctx.check(self.ctx.lib.nicp_cloud_load(self.h, str(filename).encode(),
                                                    C.byref(params) if params is not None else None, L.fptr(T),
                                                    C.byref(n)))
        self.has_stats = True
        return T.reshape(4, 4)

    def add(self, cloud, T=None):
        """Cloud::add (cloud.cpp:163-189): `cloud` is transformed in place by T
        (as the reference does) and appended to this cloud."""
        self.ctx.check(self.ctx.lib.nicp_cloud_add(self.h, cloud.h, L.fptr(L.f16(T))))
        if not cloud.has_stats:
            self.has_stats = False
        return self

    def upload(self, points, normals, curvature, omega_p=None, omega_n=None):
        n = len(points)
        p = np.ascontiguousarray(points, np.float32).reshape(n, 4)
        nn = np.ascontiguousarray(normals, np.float32).reshape(n, 4)
        k = np.ascontiguousarray(curvature, np.float32).reshape(n)
        op = None if omega_p is None else np.ascontiguousarray(omega_p, np.float32).reshape(n, 9)
        on = None if omega_n is None else np.ascontiguousarray(omega_n, np.float32).reshape(n, 9)
        self.ctx.check(self.ctx.lib.nicp_cloud_upload(self.h, n, L.fptr(p), L.fptr(nn), L.fptr(k), L.fptr(op),
                                                      L.fptr(on)))

    def transformInPlace(self, T):
        self.ctx.check(self.ctx.lib.nicp_cloud_transform(self.h, L.fptr(L.f16(T))))


# ------------------------------------------------------------------ projector
class PinholePointProjector:
    """PinholePointProjector (pinholepointprojector.{h,cpp}, pointprojector.{h,cpp}).

    Difference from the reference, by design: setImageSize() also applies the
    current scaling factor (the reference leaves imageRows()/imageCols() at
    zero until scale() is called, pointprojector.cpp:106-112)."""

    def __init__(self, ctx=None):
        self.ctx = ctx or Context.default()
        self._K = np.array([[1.0, 0.0, 0.5], [0.0, 1.0, 0.5], [0.0, 0.0, 1.0]], np.float32)
        self._transform = np.eye(4, dtype=np.float32)
        self._minDistance, self._maxDistance = 0.01, 6.0
        self._baseline, self._alpha = 0.075, 0.1
        self._rows = self._cols = 0
        self._scaling = 1.0

    # setters / getters with the reference names
    def setCameraMatrix(self, K):
        self._K = np.asarray(K, np.float32).reshape(3, 3).copy()

    def originalCameraMatrix(self):
        return self._K.copy()

    def cameraMatrix(self):
        K = self._K.copy()
        K[:2, :] *= np.float32(self._scaling)
        return K

    def setTransform(self, T):
        self._transform = np.asarray(T, np.float32).reshape(4, 4).copy()

    def transform(self):
        return self._transform.copy()

    def setMinDistance(self, v):
        self._minDistance = float(v)

    def minDistance(self):
        return self._minDistance

    def setMaxDistance(self, v):
        self._maxDistance = float(v)

    def maxDistance(self):
        return self._maxDistance

    def setBaseline(self, v):
        self._baseline = float(v)

    def setAlpha(self, v):
        self._alpha = float(v)

    def setImageSize(self, rows, cols):
        self._rows, self._cols = int(rows), int(cols)

    def scale(self, factor):
        self._scaling = float(factor)

    def scalingFactor(self):
        return self._scaling

    def imageRows(self):
        return int(np.float32(self._rows) * np.float32(self._scaling))

    def imageCols(self):
        return int(np.float32(self._cols) * np.float32(self._scaling))

    def camera(self, rows=None, cols=None):
        c = L.Camera()
        c.fx, c.fy, c.cx, c.cy = float(self._K[0, 0]), float(self._K[1, 1]), float(self._K[0, 2]), float(self._K[1, 2])
        c.scaling = self._scaling
        c.rows = self._rows if rows is None else rows
        c.cols = self._cols if cols is None else cols
        c.min_distance, c.max_distance = self._minDistance, self._maxDistance
        c.baseline, c.alpha = self._baseline, self._alpha
        return c

    def matrices(self, T=None):
        """(KRt, iKRt) of _updateMatrices() for transform T (default: transform())."""
        KRt, iKRt = np.zeros(16, np.float32), np.zeros(16, np.float32)
        c = self.camera(max(self._rows, 1), max(self._cols, 1))
        L.check(self.ctx.lib.nicp_projector_matrices(C.byref(c), L.fptr(L.f16(self._transform if T is None else T)),
                                                     L.fptr(KRt), L.fptr(iKRt)))
        return KRt.reshape(4, 4), iKRt.reshape(4, 4)

    def project(self, cloud):
        """z-buffer projection of `cloud` seen from transform(): (indexImage, depthImage)."""
        rows, cols = self.imageRows(), self.imageCols()
        if rows <= 0 or cols <= 0:
            raise ValueError("PinholePointProjector: call setImageSize() before project()")
        index = np.zeros((rows, cols), np.int32)
        depth = np.zeros((rows, cols), np.float32)
        c = self.camera()
        self.ctx.check(self.ctx.lib.nicp_project(self.ctx.h, cloud.h, C.byref(c), L.fptr(L.f16(self._transform)),
                                                 L.iptr(index), L.fptr(depth)))
        return index, depth

    def unProject(self, depthImage):
        """(points (V x 4), indexImage) of a float depth image in metres."""
        d = np.ascontiguousarray(depthImage, np.float32)
        rows, cols = d.shape
        pts = np.zeros((rows * cols, 4), np.float32)
        index = np.zeros((rows, cols), np.int32)
        n = C.c_int(0)
        c = self.camera(rows, cols)
        self.ctx.check(self.ctx.lib.nicp_unproject(self.ctx.h, L.fptr(d), rows, cols, C.byref(c),
                                                   L.fptr(L.f16(self._transform)), L.fptr(pts), L.iptr(index),
                                                   C.byref(n)))
        return pts[:n.value].copy(), index

    def projectIntervals(self, depthImage, worldRadius):
        d = np.ascontiguousarray(depthImage, np.float32)
        rows, cols = d.shape
        out = np.zeros((rows, cols), np.int32)
        c = self.camera(rows, cols)
        self.ctx.check(self.ctx.lib.nicp_project_intervals(self.ctx.h, L.fptr(d), rows, cols, C.byref(c),
                                                           float(worldRadius), L.iptr(out)))
        return np.stack([out, out], axis=-1)


# ------------------------------------------------------------------ cloud construction
class StatsCalculatorIntegralImage:
    """statscalculatorintegralimage.{h,cpp}; defaults from its constructor."""

    def __init__(self):
        self._worldRadius = 0.1
        self._maxImageRadius = 30
        self._minImageRadius = 10
        self._minPoints = 50
        self._curvatureThreshold = 0.02
        self.momentsPrecision = L.NICP_MOMENTS_F64

    def setWorldRadius(self, v): self._worldRadius = float(v)
    def worldRadius(self): return self._worldRadius
    def setMaxImageRadius(self, v): self._maxImageRadius = int(v)
    def maxImageRadius(self): return self._maxImageRadius
    def setMinImageRadius(self, v): self._minImageRadius = int(v)
    def minImageRadius(self): return self._minImageRadius
    def setMinPoints(self, v): self._minPoints = int(v)
    def minPoints(self): return self._minPoints
    def setCurvatureThreshold(self, v): self._curvatureThreshold = float(v)
    def curvatureThreshold(self): return self._curvatureThreshold


class _InformationMatrixCalculator:
    def __init__(self, flat, nonflat):
        self._flat = np.array(flat, np.float32)
        self._nonflat = np.array(nonflat, np.float32)
        self._curvatureThreshold = 0.02
        self._scale = 1.0

    def setFlatInformationMatrix(self, M):
        self._flat = np.diag(np.asarray(M, np.float32).reshape(4, 4))[:3].copy() if np.ndim(M) == 2 else \
            np.asarray(M, np.float32)[:3].copy()

    def flatInformationMatrix(self):
        M = np.zeros((4, 4), np.float32)
        M[:3, :3] = np.diag(self._flat)
        return M

    def setNonFlatInformationMatrix(self, M):
        self._nonflat = np.diag(np.asarray(M, np.float32).reshape(4, 4))[:3].copy() if np.ndim(M) == 2 else \
            np.asarray(M, np.float32)[:3].copy()

    def nonFlatInformationMatrix(self):
        M = np.zeros((4, 4), np.float32)
        M[:3, :3] = np.diag(self._nonflat)
        return M

    def setCurvatureThreshold(self, v): self._curvatureThreshold = float(v)
    def curvatureThreshold(self): return self._curvatureThreshold


class PointInformationMatrixCalculator(_InformationMatrixCalculator):
    """informationmatrixcalculator.h:115-119 defaults."""

    def __init__(self):
        super().__init__([1000.0, 0.001, 0.001], [1.0, 0.1, 0.1])


class NormalInformationMatrixCalculator(_InformationMatrixCalculator):
    """informationmatrixcalculator.h:150-155 defaults."""

    def __init__(self):
        super().__init__([1000.0, 0.001, 0.001], [0.1, 1.0, 1.0])


class DepthImageConverterIntegralImage:
    """depthimageconverterintegralimage.{h,cpp}: depth image -> Cloud on the GPU."""

    def __init__(self, projector, statsCalculator, pointInformationMatrixCalculator,
                 normalInformationMatrixCalculator):
        self._projector = projector
        self._statsCalculator = statsCalculator
        self._pim = pointInformationMatrixCalculator
        self._nim = normalInformationMatrixCalculator
        self.depthScale = 0.001
        self.keepStats = False
        # unProject's per-point Gaussian3f (mean + covariance); the reference
        # always fills Cloud::gaussians(), here it is opt-in
        self.keepGaussians = False
        self._indexImage = None

    def projector(self): return self._projector
    def setProjector(self, p): self._projector = p
    def statsCalculator(self): return self._statsCalculator
    def setStatsCalculator(self, s): self._statsCalculator = s
    def pointInformationMatrixCalculator(self): return self._pim
    def normalInformationMatrixCalculator(self): return self._nim
    def indexImage(self): return self._indexImage

    def params(self):
        s, p, n = self._statsCalculator, self._pim, self._nim
        prm = L.CloudParams()
        prm.depth_scale = self.depthScale
        prm.world_radius = s._worldRadius
        prm.min_image_radius, prm.max_image_radius, prm.min_points = s._minImageRadius, s._maxImageRadius, s._minPoints
        prm.curvature_threshold = s._curvatureThreshold
        prm.pim_flat[:] = [float(x) for x in p._flat]
        prm.pim_nonflat[:] = [float(x) for x in p._nonflat]
        prm.pim_curvature_threshold = p._curvatureThreshold
        prm.nim_flat[:] = [float(x) for x in n._flat]
        prm.nim_nonflat[:] = [float(x) for x in n._nonflat]
        prm.nim_curvature_threshold = n._curvatureThreshold
        prm.moments_precision = s.momentsPrecision
        prm.keep_stats = 1 if self.keepStats else 0
        prm.keep_gaussians = 1 if self.keepGaussians else 0
        return prm

    def compute(self, cloud, depthImage, sensorOffset=None, keep_index=False):
        """uint16 (millimetres, scaled by depthScale) or float32 (metres) depth."""
        d = np.ascontiguousarray(depthImage)
        rows, cols = d.shape
        self._projector.setImageSize(rows, cols)
        # the converter unprojects in the camera frame and leaves the
        # projector there (depthimageconverterintegralimage.cpp:42)
        self._projector.setTransform(np.eye(4))
        cam = self._projector.camera(rows, cols)
        prm = self.params()
        idx = np.zeros((rows, cols), np.int32) if keep_index else None
        off = L.fptr(L.f16(sensorOffset)) if sensorOffset is not None else None
        ctx = cloud.ctx
        if d.dtype == np.uint16:
            fn = ctx.lib.nicp_cloud_from_depth_u16
        elif d.dtype == np.float32:
            fn = ctx.lib.nicp_cloud_from_depth_f32
        else:
            raise TypeError("depth must be uint16 or float32")
        ctx.check(fn(ctx.h, d.ctypes.data_as(C.c_void_p), rows, cols, 0, 0, C.byref(cam), C.byref(prm), off, cloud.h,
                     L.iptr(idx)))
        cloud.has_stats = self.keepStats
        self._indexImage = idx
        return cloud


# ------------------------------------------------------------------ registration
def trajectory_line(timestamp, T):
    """A line of nicp_simple_aligner's trajectory file (lines 175-181):
    "timestamp tx ty tz qx qy qz qw"."""
    buf = C.create_string_buffer(512)
    L.check(L.load().nicp_trajectory_line(str(timestamp).encode(), L.fptr(L.f16(T)), buf, len(buf)))
    return buf.value.decode()


def DepthImage_scale(depth, step, maxDepthCov=0.01, depthScale=0.001, ctx=None):
    """DepthImage_scale (imageutils.cpp:6-37) on the GPU: a (rows/step) x
    (cols/step) float image (metres), each pixel the mean of its block's
    positive depths, 0 when the block has none or their variance exceeds
    maxDepthCov.  `depth`: uint16 (times depthScale, i.e. with
    DepthImage_convert_16UC1_to_32FC1 fused in front) or float32 metres.
    Use it with a projector scaled by 1/step (PinholePointProjector.scale)."""
    ctx = ctx or Context.default()
    d = np.ascontiguousarray(depth)
    if d.dtype not in (np.uint16, np.float32):
        raise TypeError("depth must be uint16 or float32")
    rows, cols = d.shape
    out = np.zeros((rows // step, cols // step), np.float32)
    ctx.check(ctx.lib.nicp_depth_scale(ctx.h, d.ctypes.data_as(C.c_void_p), 1 if d.dtype == np.uint16 else 0, rows,
                                       cols, 0, 0, float(depthScale), int(step), float(maxDepthCov),
                                       out.ctypes.data_as(C.c_void_p), 0))
    return out


def DepthImage_convert_16UC1_to_32FC1(depth_u16, scale=0.001, ctx=None):
    """imageutils.cpp:85-99 on the GPU: u16 -> float metres (0 stays 0)."""
    return DepthImage_scale(np.ascontiguousarray(depth_u16, np.uint16), 1, 0.01, scale, ctx)


class Merger:
    """merger.{h,cpp}: fuses the points of a cloud that land on the same pixel
    of a view (Gaussian information fusion) and removes the absorbed ones.
    Defaults merger.cpp:5-13.  The cloud needs Gaussians (a converter with
    keepGaussians = True)."""

    def __init__(self, ctx=None):
        self.ctx = ctx or Context.default()
        self._distanceThreshold = 0.1
        self._normalThreshold = float(np.float32(math.cos(10 * math.pi / 180.0)))  # kept, unused by merge()
        self._maxPointDepth = 10.0
        self._depthImageConverter = None
        self._rows = self._cols = 0
        self.removed = 0

    def distanceThreshold(self): return self._distanceThreshold
    def setDistanceThreshold(self, v): self._distanceThreshold = float(v)
    def normalThreshold(self): return self._normalThreshold
    def setNormalThreshold(self, v): self._normalThreshold = float(v)
    def maxPointDepth(self): return self._maxPointDepth
    def setMaxPointDepth(self, v): self._maxPointDepth = float(v)
    def depthImageConverter(self): return self._depthImageConverter
    def setDepthImageConverter(self, c): self._depthImageConverter = c
    def imageSize(self): return (self._rows, self._cols)

    def setImageSize(self, r, c):
        self._rows, self._cols = int(r), int(c)

    def merge(self, cloud, transform=None):
        if self._rows <= 0 or self._cols <= 0:
            raise ValueError("Merger: call setImageSize() first")
        if self._depthImageConverter is None:
            raise ValueError("Merger: missing depth image converter")
        cam = self._depthImageConverter.projector().camera(self._rows, self._cols)
        removed = C.c_int(0)
        T = np.eye(4, dtype=np.float32) if transform is None else transform
        self.ctx.check(self.ctx.lib.nicp_merge(self.ctx.h, cloud.h, C.byref(cam), L.fptr(L.f16(T)),
                                               self._distanceThreshold, self._maxPointDepth, C.byref(removed)))
        self.removed = removed.value
        return cloud


class CorrespondenceFinderProjective:
    """correspondencefinder{,projective}.{h,cpp}; defaults correspondencefinder.cpp:9-18."""

    def __init__(self, ctx=None):
        self.ctx = ctx or Context.default()
        self._inlierDistanceThreshold = 1.0
        self._inlierNormalAngularThreshold = float(np.float32(math.cos(np.float32(math.pi / 6))))
        self._flatCurvatureThreshold = 0.2
        self._inlierCurvatureRatioThreshold = 1.3
        self._demotedToGICP = False
        self._rows = self._cols = 0
        self.parityThreads = 1
        self._rowSearchRegion = self._colSearchRegion = 0  # correspondencefinderprojective.cpp:12-13
        self._referenceIndexImage = None
        self._currentIndexImage = None
        self._referenceDepthImage = None
        self._currentDepthImage = None
        self._correspondences = np.zeros((0, 2), np.int32)

    def setInlierDistanceThreshold(self, v): self._inlierDistanceThreshold = float(v)
    def inlierDistanceThreshold(self): return self._inlierDistanceThreshold
    def squaredThreshold(self): return float(np.float32(self._inlierDistanceThreshold) ** 2)
    def setInlierNormalAngularThreshold(self, v): self._inlierNormalAngularThreshold = float(v)
    def inlierNormalAngularThreshold(self): return self._inlierNormalAngularThreshold
    def setFlatCurvatureThreshold(self, v): self._flatCurvatureThreshold = float(v)
    def flatCurvatureThreshold(self): return self._flatCurvatureThreshold
    def setInlierCurvatureRatioThreshold(self, v): self._inlierCurvatureRatioThreshold = float(v)
    def inlierCurvatureRatioThreshold(self): return self._inlierCurvatureRatioThreshold
    def setDemotedToGICP(self, v): self._demotedToGICP = bool(v)
    # correspondencefinderprojective.h:146-150: a search window (0 0 = the pixel itself)
    def rowSearchRegion(self): return self._rowSearchRegion
    def colSearchRegion(self): return self._colSearchRegion
    def setRowSearchRegion(self, v): self._rowSearchRegion = int(v)
    def setColSearchRegion(self, v): self._colSearchRegion = int(v)
    def demotedToGICP_(self): return self._demotedToGICP
    def setImageSize(self, rows, cols): self._rows, self._cols = int(rows), int(cols)
    def imageRows(self): return self._rows
    def imageCols(self): return self._cols
    def referenceIndexImage(self): return self._referenceIndexImage
    def currentIndexImage(self): return self._currentIndexImage
    def setReferenceIndexImage(self, im): self._referenceIndexImage = np.ascontiguousarray(im, np.int32)
    def setCurrentIndexImage(self, im): self._currentIndexImage = np.ascontiguousarray(im, np.int32)
    def correspondences(self): return self._correspondences
    def numCorrespondences(self): return len(self._correspondences)

    def params(self):
        p = L.CorrParams()
        p.inlier_distance_threshold = self._inlierDistanceThreshold
        p.inlier_normal_angular_threshold = self._inlierNormalAngularThreshold
        p.flat_curvature_threshold = self._flatCurvatureThreshold
        p.inlier_curvature_ratio_threshold = self._inlierCurvatureRatioThreshold
        p.demoted_to_gicp = 1 if self._demotedToGICP else 0
        p.parity_threads = self.parityThreads
        p.row_search_region = self._rowSearchRegion
        p.col_search_region = self._colSearchRegion
        return p

    def compute(self, referenceScene, currentScene, T):
        ri, ci = self._referenceIndexImage, self._currentIndexImage
        if ri is None or ci is None:
            raise ValueError("CorrespondenceFinderProjective: index images are not set")
        rows, cols = ri.shape
        pairs = np.zeros((rows * cols, 2), np.int32)
        k = C.c_int(0)
        p = self.params()
        self.ctx.check(self.ctx.lib.nicp_correspond(self.ctx.h, referenceScene.h, currentScene.h, L.iptr(ri),
                                                    L.iptr(ci), rows, cols, L.fptr(L.f16(T)), C.byref(p),
                                                    L.iptr(pairs), C.byref(k)))
        self._correspondences = pairs[:k.value].copy()
        return self._correspondences


class Linearizer:
    """linearizer.{h,cpp}; defaults linearizer.cpp:9-19.  update() (alias
    linearize()) builds H, b, error and inliers over the aligner's current
    correspondences, accumulated in FP64."""

    def __init__(self, ctx=None):
        self.ctx = ctx or Context.default()
        self._aligner = None
        self._T = np.eye(4, dtype=np.float32)
        self._inlierMaxChi2 = 9e3
        self._robustKernel = True
        self._demotedToGeneralizedICP = False
        # precision study: sum the per-tile partials in FP32 (default FP64)
        self.crossBlockF32 = False
        self._zScaling = False
        self._scale = 1.0
        self._H = np.zeros((6, 6))
        self._b = np.zeros(6)
        self._error = 0.0
        self._inliers = 0

    def setAligner(self, a): self._aligner = a
    def aligner(self): return self._aligner
    def setT(self, T):
        self._T = np.asarray(T, np.float32).reshape(4, 4).copy()
        self._T[3] = [0, 0, 0, 1]
    def T(self): return self._T.copy()
    def setInlierMaxChi2(self, v): self._inlierMaxChi2 = float(v)
    def inlierMaxChi2(self): return self._inlierMaxChi2
    def setRobustKernel(self, v): self._robustKernel = bool(v)
    def robustKernel(self): return self._robustKernel
    def setDemotedToGeneralizedICP(self, v): self._demotedToGeneralizedICP = bool(v)
    def demotedToGeneralizedICP(self): return self._demotedToGeneralizedICP
    def setZScaling(self, v): self._zScaling = bool(v)
    def zScaling(self): return self._zScaling
    def setScale(self, v): self._scale = float(v)
    def scale(self): return self._scale
    def H(self): return self._H.copy()
    def b(self): return self._b.copy()
    def error(self): return self._error
    def inliers(self): return self._inliers

    def params(self):
        p = L.LinParams()
        p.inlier_max_chi2 = self._inlierMaxChi2
        p.robust_kernel = 1 if self._robustKernel else 0
        p.z_scaling = 1 if self._zScaling else 0
        p.scale = self._scale
        p.demoted_to_gicp = 1 if self._demotedToGeneralizedICP else 0
        p.cross_block_f32 = 1 if self.crossBlockF32 else 0
        return p

    def update(self, referenceCloud=None, currentCloud=None, correspondences=None, parity_threads=None):
        a = self._aligner
        ref = referenceCloud or a.referenceCloud()
        cur = currentCloud or a.currentCloud()
        cf = a.correspondenceFinder() if a is not None else None
        pairs = correspondences if correspondences is not None else cf.correspondences()
        pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        T = parity_threads if parity_threads is not None else (cf.parityThreads if cf is not None else 1)
        H, b, err = np.zeros(36), np.zeros(6), C.c_double(0)
        inl = C.c_int(0)
        p = self.params()
        self.ctx.check(self.ctx.lib.nicp_linearize(self.ctx.h, ref.h, cur.h, L.iptr(pairs), len(pairs),
                                                   L.fptr(L.f16(self._T)), C.byref(p), int(T), L.dptr(H), L.dptr(b),
                                                   C.byref(err), C.byref(inl)))
        self._H, self._b, self._error, self._inliers = H.reshape(6, 6), b, err.value, inl.value

    linearize = update


class AlignerProjective:
    """aligner.{h,cpp} + alignerprojective.{h,cpp}: the whole outer x inner
    Gauss-Newton loop runs on the device (FP64 6x6 LDL^T solve and pose update)
    with one host synchronisation at the end of align()."""

    def __init__(self, projector=None, linearizer=None, correspondenceFinder=None, ctx=None):
        self.ctx = ctx or Context.default()
        self._projector = projector
        self._linearizer = None
        self._correspondenceFinder = correspondenceFinder
        if linearizer is not None:
            self.setLinearizer(linearizer)
        self._referenceCloud = self._currentCloud = None
        self._outerIterations, self._innerIterations = 10, 1
        self._T = np.eye(4)
        self._initialGuess = np.eye(4, dtype=np.float32)
        self._referenceSensorOffset = np.eye(4, dtype=np.float32)
        self._currentSensorOffset = np.eye(4, dtype=np.float32)
        self._totalTime = 0.0
        self._error = 0.0
        self._inliers = 0
        self._minInliers = 100
        self._rotationalMinEigenRatio = 50.0
        self._translationalMinEigenRatio = 50.0
        self._lambda = 1e3
        self._debug = False
        self._solutionValid = False
        self._translationalEigenRatio = self._rotationalEigenRatio = 0.0
        self._omega = np.zeros((6, 6))
        self._mean = np.zeros(6)
        self.computeStatistics = True
        self.earlyExitEps = 0.0
        self.last_result = None

    def projector(self): return self._projector
    def setProjector(self, p): self._projector = p
    def linearizer(self): return self._linearizer

    def setLinearizer(self, lin):
        self._linearizer = lin
        lin.setAligner(self)  # aligner.h:212-216

    def correspondenceFinder(self): return self._correspondenceFinder
    def setCorrespondenceFinder(self, cf): self._correspondenceFinder = cf
    def referenceCloud(self): return self._referenceCloud
    def setReferenceCloud(self, c): self._referenceCloud = c
    def currentCloud(self): return self._currentCloud
    def setCurrentCloud(self, c): self._currentCloud = c
    def outerIterations(self): return self._outerIterations
    def setOuterIterations(self, v): self._outerIterations = int(v)
    def innerIterations(self): return self._innerIterations
    def setInnerIterations(self, v): self._innerIterations = int(v)
    def T(self): return self._T.copy()
    def initialGuess(self): return self._initialGuess.copy()
    def setInitialGuess(self, T): self._initialGuess = np.asarray(T, np.float32).reshape(4, 4).copy()

    def setSensorOffset(self, T):
        self._referenceSensorOffset = np.asarray(T, np.float32).reshape(4, 4).copy()
        self._currentSensorOffset = self._referenceSensorOffset.copy()

    def sensorOffset(self): return self._referenceSensorOffset.copy()
    def setReferenceSensorOffset(self, T): self._referenceSensorOffset = np.asarray(T, np.float32).reshape(4, 4).copy()
    def referenceSensorOffset(self): return self._referenceSensorOffset.copy()
    def setCurrentSensorOffset(self, T): self._currentSensorOffset = np.asarray(T, np.float32).reshape(4, 4).copy()
    def currentSensorOffset(self): return self._currentSensorOffset.copy()
    def setDebug(self, v): self._debug = bool(v)
    def debug(self): return self._debug
    def setMinInliers(self, v): self._minInliers = int(v)
    def minInliers(self): return self._minInliers
    def setTranslationalMinEigenRatio(self, v): self._translationalMinEigenRatio = float(v)
    def translationalMinEigenRatio(self): return self._translationalMinEigenRatio
    def setRotationalMinEigenRatio(self, v): self._rotationalMinEigenRatio = float(v)
    def rotationalMinEigenRatio(self): return self._rotationalMinEigenRatio
    def translationalEigenRatio(self): return self._translationalEigenRatio
    def rotationalEigenRatio(self): return self._rotationalEigenRatio
    def setLambda(self, v): self._lambda = float(v)
    def lambda_(self): return self._lambda
    def solutionValid(self): return self._solutionValid
    def omega(self): return self._omega.copy()  # aligner.h:325, 6x6 in (t, quaternion-vector)
    def mean(self): return self._mean.copy()
    def error(self): return self._error
    def inliers(self): return self._inliers
    def totalTime(self): return self._totalTime

    def params(self):
        p = L.AlignParams()
        p.outer_iterations, p.inner_iterations = self._outerIterations, self._innerIterations
        p.lambda_ = self._lambda
        p.min_inliers = self._minInliers
        p.translational_min_eigen_ratio = self._translationalMinEigenRatio
        p.rotational_min_eigen_ratio = self._rotationalMinEigenRatio
        p.compute_statistics = 1 if self.computeStatistics else 0
        p.early_exit_eps = self.earlyExitEps
        return p

    def align(self):
        import time
        proj, lin, cf = self._projector, self._linearizer, self._correspondenceFinder
        if proj is None or lin is None or cf is None:
            raise ValueError("AlignerProjective: projector, linearizer and correspondence finder must be set")
        if self._referenceCloud is None or self._currentCloud is None:
            raise ValueError("AlignerProjective: reference and current clouds must be set")
        cam = proj.camera()
        if cam.rows <= 0 or cam.cols <= 0:
            raise ValueError("AlignerProjective: the projector has no image size")
        r = L.AlignResult()
        cp, lp, ap = cf.params(), lin.params(), self.params()
        t0 = time.perf_counter()
        self.ctx.check(self.ctx.lib.nicp_align(self.ctx.h, self._referenceCloud.h, self._currentCloud.h,
                                               C.byref(cam), L.fptr(L.f16(self._initialGuess)),
                                               L.fptr(L.f16(self._referenceSensorOffset)),
                                               L.fptr(L.f16(self._currentSensorOffset)), C.byref(cp), C.byref(lp),
                                               C.byref(ap), C.byref(r)))
        self._totalTime = (time.perf_counter() - t0) * 1e3
        self._T = np.array(r.T).reshape(4, 4)
        self._error = r.error
        self._inliers = r.inliers
        lin._error, lin._inliers = r.error, r.inliers
        self._translationalEigenRatio = r.translational_ratio
        self._rotationalEigenRatio = r.rotational_ratio
        self._solutionValid = bool(r.solution_valid == 1)
        self._omega = np.array(r.omega).reshape(6, 6)
        self._mean = np.array(r.mean)
        self.last_result = r
        return self._T


class CorrespondenceFinderNN(CorrespondenceFinderProjective):
    """correspondencefindernn.{h,cpp}: nearest neighbour in (p, s n) within
    the inlier distance, then the normal gates.  The search is exact (ties:
    lowest index) where the reference's FLANN kd-tree is approximate."""

    def __init__(self, ctx=None):
        super().__init__(ctx)
        self._normalScaling = 1.0  # correspondencefindernn.cpp:5-9

    def normalScaling(self): return self._normalScaling
    def setNormalScaling(self, v): self._normalScaling = float(v)

    def compute(self, referenceScene, currentScene, T):
        n = referenceScene.size()
        pairs = np.zeros((max(n, 1), 2), np.int32)
        k = C.c_int(0)
        self.ctx.check(self.ctx.lib.nicp_correspond_nn(self.ctx.h, referenceScene.h, currentScene.h,
                                                       L.fptr(L.f16(T)), self._normalScaling,
                                                       C.byref(self.params()), L.iptr(pairs), C.byref(k)))
        self._correspondences = pairs[:k.value].copy()
        return self._correspondences


class AlignerNN(AlignerProjective):
    """alignernn.{h,cpp}: AlignerProjective's loop with nearest-neighbour
    correspondences (CorrespondenceFinderNN); needs no projector."""

    def align(self):
        import time
        lin, cf = self._linearizer, self._correspondenceFinder
        if lin is None or not isinstance(cf, CorrespondenceFinderNN):
            raise ValueError("AlignerNN: a linearizer and a CorrespondenceFinderNN must be set")
        if self._referenceCloud is None or self._currentCloud is None:
            raise ValueError("AlignerNN: reference and current clouds must be set")
        r = L.AlignResult()
        t0 = time.perf_counter()
        self.ctx.check(self.ctx.lib.nicp_align_nn(self.ctx.h, self._referenceCloud.h, self._currentCloud.h,
                                                  L.fptr(L.f16(self._initialGuess)), cf.normalScaling(),
                                                  C.byref(cf.params()), C.byref(lin.params()), C.byref(self.params()),
                                                  C.byref(r)))
        self._totalTime = (time.perf_counter() - t0) * 1e3
        self._T = np.array(r.T).reshape(4, 4)
        self._error = r.error
        self._inliers = r.inliers
        lin._error, lin._inliers = r.error, r.inliers
        self._translationalEigenRatio = r.translational_ratio
        self._rotationalEigenRatio = r.rotational_ratio
        self._solutionValid = bool(r.solution_valid == 1)
        self._omega = np.array(r.omega).reshape(6, 6)
        self._mean = np.array(r.mean)
        self.last_result = r
        return self._T


# ------------------------------------------------------------------ batching (no reference counterpart)
def build_batch(ctx, frames, cams, prm, clouds, on_device=False):
    """Builds clouds for many uint16 frames in one pass of launches.  frames:
    list of host arrays, or of device pointers (ints) with on_device=True."""
    n = len(frames)
    ptrs = (C.c_void_p * n)()
    rows = np.zeros(n, np.int32)
    cols = np.zeros(n, np.int32)
    keep = []
    for i, f in enumerate(frames):
        if on_device:
            ptrs[i] = f[0]
            rows[i], cols[i] = f[1], f[2]
        else:
            a = np.ascontiguousarray(f, np.uint16)
            keep.append(a)
            ptrs[i] = a.ctypes.data
            rows[i], cols[i] = a.shape
    camarr = (L.Camera * n)(*cams)
    outs = (C.c_void_p * n)(*[c.h.value for c in clouds])
    ctx.check(ctx.lib.nicp_build_batch(ctx.h, n, ptrs, L.iptr(rows), L.iptr(cols), 1 if on_device else 0, camarr,
                                       C.byref(prm), outs))
    return clouds


def align_batch(ctx, refs, curs, cams, guesses, corr, lin, prm):
    n = len(refs)
    r = (C.c_void_p * n)(*[c.h.value for c in refs])
    c = (C.c_void_p * n)(*[x.h.value for x in curs])
    camarr = (L.Camera * n)(*cams)
    g = None
    if guesses is not None:
        g = np.ascontiguousarray(np.asarray(guesses, np.float32).reshape(n, 16))
    res = (L.AlignResult * n)()
    ctx.check(ctx.lib.nicp_align_batch(ctx.h, n, r, c, camarr, L.fptr(g), C.byref(corr), C.byref(lin), C.byref(prm),
                                       res))
    return res


# ------------------------------------------------------------------ serving (no reference counterpart)
class Server:
    """Continuous-batching request loop (nicp_server_* in include/nicp_gpu.h):
    device-resident keyframe per camera stream, admission by HBM budget,
    batches formed as requests arrive, several batches in flight."""

    def __init__(self, device=0, hbm_budget_bytes=60 << 30, max_batch=64, workers=2, keyframe_min_inlier_ratio=0.4,
                 params=None):
        self.lib = L.load()
        p = L.ServerParams()
        self.lib.nicp_default_server_params(C.byref(p))
        p.hbm_budget_bytes = int(hbm_budget_bytes)
        p.max_batch, p.workers = int(max_batch), int(workers)
        p.keyframe_min_inlier_ratio = float(keyframe_min_inlier_ratio)
        if params:
            params(p)
        h = C.c_void_p()
        rc = self.lib.nicp_server_create(device, C.byref(p), C.byref(h))
        if rc != L.NICP_OK:
            raise L.NicpError(rc, "cannot create the server")
        self.h = h
        self._buf = (L.ServerResult * 4096)()

    def submit(self, stream_id, request_id, depth_u16, camera):
        d = np.ascontiguousarray(depth_u16, np.uint16)
        rows, cols = d.shape
        rc = self.lib.nicp_server_submit(self.h, int(stream_id), int(request_id), d.ctypes.data_as(C.c_void_p),
                                         rows, cols, C.byref(camera))
        L.check(rc)

    def poll(self, wait_ms=0):
        n = C.c_int(0)
        L.check(self.lib.nicp_server_poll(self.h, self._buf, len(self._buf), C.byref(n), int(wait_ms)))
        out = []
        for i in range(n.value):
            r = self._buf[i]
            out.append(dict(request_id=r.request_id, stream_id=r.stream_id, status=r.status,
                            T=np.array(r.T).reshape(4, 4), error=r.error, inliers=r.inliers,
                            keyframe_points=r.keyframe_points, keyframe_replaced=bool(r.keyframe_replaced),
                            batch_size=r.batch_size, latency_ms=r.latency_ms, queue_ms=r.queue_ms))
        return out

    def status(self):
        p, b = C.c_int(0), C.c_size_t(0)
        L.check(self.lib.nicp_server_status(self.h, C.byref(p), C.byref(b)))
        return p.value, b.value

    def drain(self, expected, timeout_s=120.0):
        import time
        got, t0 = [], time.time()
        while len(got) < expected and time.time() - t0 < timeout_s:
            got += self.poll(wait_ms=50)
        return got

    def close(self):
        if getattr(self, "h", None):
            self.lib.nicp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
