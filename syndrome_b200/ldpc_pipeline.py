"""src/ldpc_pipeline.rs LdpcPipeline on the GPU: acquire a frame, fill its N f32
LLRs, submit it, receive it decoded (decode_layered_offset_min_sum: its LLRs become
the posterior, with hard decisions and the iterations used), release it.

Host worker threads batch the submitted frames into one f32 decode launch each on
their own CUDA streams; frames live in pinned host memory, so `llr_mut()` and
`hard()` are numpy views of it."""
import ctypes

import numpy as np

from . import _lib


class LdpcFrame:
    """One frame of a pipeline's pool (ldpc_pipeline.rs:157-228)."""

    def __init__(self, pipe, index):
        self._p = pipe
        self.index = int(index)

    def llr_mut(self):
        L = _lib.load()
        ptr = L.syndrome_ldpc_pipeline_frame_llr(self._p._h, self.index)
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), shape=(self._p.n,))

    def hard(self):
        L = _lib.load()
        ptr = L.syndrome_ldpc_pipeline_frame_hard(self._p._h, self.index)
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)), shape=(self._p.n,))

    def iterations_used(self):
        return int(_lib.load().syndrome_ldpc_pipeline_frame_iterations(self._p._h, self.index))

    def set_tag(self, tag):
        _lib.load().syndrome_ldpc_pipeline_frame_set_tag(self._p._h, self.index, int(tag))

    def tag(self):
        return int(_lib.load().syndrome_ldpc_pipeline_frame_tag(self._p._h, self.index))


class LdpcPipeline:
    """ldpc_pipeline.rs:288-598.  `decoder` (a QcLdpcDecoder) must outlive the pipeline."""

    def __init__(self, decoder, iterations, n_workers=0):
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_ldpc_pipeline_create(decoder._h, int(iterations), int(n_workers),
                                                            ctypes.byref(h)))
        self._h = h.value
        self._decoder = decoder  # keeps the decoder alive
        self.n = decoder.variable_node_count()

    @classmethod
    def new(cls, decoder, iterations):
        return cls(decoder, iterations, 0)

    @classmethod
    def with_workers(cls, decoder, iterations, n_workers):
        return cls(decoder, iterations, max(int(n_workers), 1))

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.load().syndrome_ldpc_pipeline_destroy(h)
            except Exception:
                pass

    def worker_count(self):
        return int(_lib.load().syndrome_ldpc_pipeline_worker_count(self._h))

    def pool_size(self):
        return int(_lib.load().syndrome_ldpc_pipeline_pool_size(self._h))

    def acquire(self):
        """A free frame, or None when every frame is in use."""
        f = _lib.load().syndrome_ldpc_pipeline_acquire(self._h)
        return None if f < 0 else LdpcFrame(self, f)

    def submit(self, frame):
        _lib.check(_lib.load().syndrome_ldpc_pipeline_submit(self._h, frame.index))

    def try_recv(self):
        """A decoded frame (completion order), or None."""
        f = _lib.load().syndrome_ldpc_pipeline_try_recv(self._h)
        return None if f < 0 else LdpcFrame(self, f)

    def release(self, frame):
        _lib.check(_lib.load().syndrome_ldpc_pipeline_release(self._h, frame.index))
