"""ctypes loader of oracle/_ref/librefcuda.so (elsa's own CUDA projector kernels behind the host
harness refcuda.cu; built by oracle/ref_cuda/build.py). TEST INFRASTRUCTURE ONLY."""
import ctypes
import os

# built by oracle/ref_cuda/build.py (not imported here, so that `python -m` runs it cleanly)
LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "_ref",
                   "librefcuda.so")

SYMBOLS = ["refcuda_last_error", "refcuda_create", "refcuda_destroy",
           "refcuda_joseph_upload_volume", "refcuda_joseph_forward",
           "refcuda_joseph_download_sinogram", "refcuda_joseph_upload_sinogram",
           "refcuda_joseph_adjoint_fast", "refcuda_joseph_download_volume",
           "refcuda_siddon_forward", "refcuda_siddon_adjoint", "refcuda_voxel_set_lut",
           "refcuda_voxel_forward", "refcuda_voxel_adjoint", "refcuda2d_create",
           "refcuda2d_destroy", "refcuda2d_joseph_adjoint_fast"]

_lib = None


def built():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        vp, i32, f = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float
        L.refcuda_last_error.restype = ctypes.c_char_p
        L.refcuda_create.argtypes = [vp, vp, vp, ctypes.POINTER(vp)]
        L.refcuda_destroy.argtypes = [vp]
        for name in ("refcuda_joseph_forward", "refcuda_joseph_adjoint_fast"):
            getattr(L, name).argtypes = [vp]
        for name in ("refcuda_joseph_upload_volume", "refcuda_joseph_download_sinogram",
                     "refcuda_joseph_upload_sinogram", "refcuda_joseph_download_volume"):
            getattr(L, name).argtypes = [vp, vp]
        L.refcuda_siddon_forward.argtypes = [vp, vp, vp]
        L.refcuda_siddon_adjoint.argtypes = [vp, vp, vp]
        L.refcuda_voxel_set_lut.argtypes = [vp, vp, i32, f]
        L.refcuda_voxel_forward.argtypes = [vp, i32, vp, vp]
        L.refcuda_voxel_adjoint.argtypes = [vp, i32, vp, vp]
        L.refcuda2d_create.argtypes = [vp, vp, vp, ctypes.POINTER(vp)]
        L.refcuda2d_destroy.argtypes = [vp]
        L.refcuda2d_joseph_adjoint_fast.argtypes = [vp, vp, vp]
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise RuntimeError(lib().refcuda_last_error().decode())


class RefProjectors:
    """The reference's CUDA operators for one 3D geometry (device pointers in and out; every
    call is asynchronous on the legacy default stream, the voxel projectors synchronize)."""

    def __init__(self, vol, det, poses):
        import numpy as np
        self._keep = (np.ascontiguousarray(vol, np.int64), np.ascontiguousarray(det, np.int64),
                      np.ascontiguousarray(poses, np.float32))
        h = ctypes.c_void_p()
        check(lib().refcuda_create(self._keep[0].ctypes.data, self._keep[1].ctypes.data,
                                   self._keep[2].ctypes.data, ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().refcuda_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # Joseph: texture upload + forward kernel + copy out of the pitched sinogram
    def joseph_forward(self, x_ptr, y_ptr, kernel_only=False):
        L = lib()
        if not kernel_only:
            check(L.refcuda_joseph_upload_volume(self.h, x_ptr))
        check(L.refcuda_joseph_forward(self.h))
        if not kernel_only:
            check(L.refcuda_joseph_download_sinogram(self.h, y_ptr))

    def joseph_adjoint_fast(self, y_ptr, x_ptr, kernel_only=False):
        L = lib()
        if not kernel_only:
            check(L.refcuda_joseph_upload_sinogram(self.h, y_ptr))
        check(L.refcuda_joseph_adjoint_fast(self.h))
        if not kernel_only:
            check(L.refcuda_joseph_download_volume(self.h, x_ptr))

    def siddon_forward(self, x_ptr, y_ptr):
        check(lib().refcuda_siddon_forward(self.h, x_ptr, y_ptr))

    def siddon_adjoint(self, y_ptr, x_ptr):
        check(lib().refcuda_siddon_adjoint(self.h, y_ptr, x_ptr))

    def set_lut(self, lut, radius):
        import numpy as np
        self._lut = np.ascontiguousarray(lut, np.float32)
        check(lib().refcuda_voxel_set_lut(self.h, self._lut.ctypes.data, self._lut.size,
                                          float(radius)))

    def voxel_forward(self, x_ptr, y_ptr, differential=False):
        check(lib().refcuda_voxel_forward(self.h, int(differential), x_ptr, y_ptr))

    def voxel_adjoint(self, y_ptr, x_ptr, differential=False):
        check(lib().refcuda_voxel_adjoint(self.h, int(differential), y_ptr, x_ptr))


class RefJoseph2D:
    """The reference's 2D Joseph `fast` adjoint (TraverseJosephsCUDA<float, 2>) for one fan-beam
    geometry (device pointers in and out, legacy default stream)."""

    def __init__(self, vol, det, poses):
        import numpy as np
        self._keep = (np.ascontiguousarray(vol, np.int64), np.ascontiguousarray(det, np.int64),
                      np.ascontiguousarray(poses, np.float32))
        h = ctypes.c_void_p()
        check(lib().refcuda2d_create(self._keep[0].ctypes.data, self._keep[1].ctypes.data,
                                     self._keep[2].ctypes.data, ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().refcuda2d_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def joseph_adjoint_fast(self, y_ptr, x_ptr):
        check(lib().refcuda2d_joseph_adjoint_fast(self.h, y_ptr, x_ptr))
