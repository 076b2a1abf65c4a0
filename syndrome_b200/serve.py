"""Transport-block serving on the GPU: continuous batching of DL-SCH transmissions with
device-resident HARQ accumulators (include/syndrome_ldpc.h section 5).

Per transmission the results are those of syndrome's DlSchDecoder::decode
(src/transport_block.rs:829) with the int8 code-block decode; the engine replaces the
reference's LdpcPipeline worker threads (src/ldpc_pipeline.rs) with one GPU work queue
fed by a worker thread that batches whatever has arrived."""
import ctypes

import numpy as np

from . import _lib


class _Config(ctypes.Structure):
    _fields_ = [("max_step_code_blocks", ctypes.c_uint32), ("steps_in_flight", ctypes.c_uint32),
                ("harq_bytes", ctypes.c_uint64), ("staging_bytes", ctypes.c_uint64), ("iterations", ctypes.c_int32),
                ("offset_beta", ctypes.c_float), ("scale", ctypes.c_float), ("app_clamp", ctypes.c_int32),
                ("latency_steps", ctypes.c_uint32), ("backlog_code_blocks", ctypes.c_uint32),
                ("decode_kernel", ctypes.c_int32), ("engine", ctypes.c_int32), ("idle_us", ctypes.c_uint32)]


class _Result(ctypes.Structure):
    _fields_ = [("tb_id", ctypes.c_uint64), ("crc_ok", ctypes.c_int32), ("max_iters_used", ctypes.c_int32),
                ("harq_tx_count", ctypes.c_int32), ("num_code_blocks", ctypes.c_int32),
                ("cb_crc", ctypes.c_uint32 * 5), ("reserved", ctypes.c_uint32), ("latency_us", ctypes.c_double)]


class _LoadTb(ctypes.Structure):
    _fields_ = [("tb_size", ctypes.c_size_t), ("target_rate", ctypes.c_float), ("qm", ctypes.c_size_t),
                ("g", ctypes.c_size_t), ("llr", ctypes.c_void_p * 4), ("llr_len", ctypes.c_size_t)]


class _LoadSpec(ctypes.Structure):
    _fields_ = [("offered_tb_per_s", ctypes.c_double), ("duration_s", ctypes.c_double),
                ("max_transmissions", ctypes.c_uint32), ("seed", ctypes.c_uint64)]


class _LoadReport(ctypes.Structure):
    _fields_ = [("tbs", ctypes.c_uint64), ("tbs_ok", ctypes.c_uint64), ("transmissions", ctypes.c_uint64),
                ("wall_s", ctypes.c_double), ("info_bits_ok", ctypes.c_double),
                ("info_bits_decoded", ctypes.c_double), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("max_us", ctypes.c_double),
                ("tx_p50_us", ctypes.c_double), ("tx_p99_us", ctypes.c_double),
                ("tx_mean_queue_us", ctypes.c_double), ("tx_mean_step_us", ctypes.c_double)]


class Server:
    """A serving engine on the current CUDA device.  Zero-valued sizes take the
    library defaults (2048 code blocks per step, 6 steps in flight, 8 GiB of HARQ
    accumulators, 256 MiB of staging for host-memory LLRs).

    engine="continuous" (default): one persistent kernel takes each transmission's
    code blocks as soon as they are submitted (it holds max_step_code_blocks x
    steps_in_flight code blocks in flight, exits after idle_us without work, 0 = 2000,
    and is relaunched with the next transmission); it needs kernel="auto" and
    app_clamp >= 7874, else the step engine runs.  engine="steps": batches of up to
    max_step_code_blocks, up to steps_in_flight at once (latency_steps and
    backlog_code_blocks set how many while few code blocks wait).  Results are
    identical either way; the continuous engine has the shorter latency, the step
    engine the higher saturated throughput."""

    def __init__(self, max_step_code_blocks=0, steps_in_flight=0, harq_bytes=0, staging_bytes=0, iterations=8,
                 offset_beta=0.5, scale=8.0, app_clamp=32767, latency_steps=0, backlog_code_blocks=0,
                 kernel="auto", engine="continuous", idle_us=0):
        code = {"auto": 0, "pair_smem": 5}.get(kernel)
        if code is None:
            raise ValueError(f"unknown serving kernel {kernel!r}")
        mode = {"continuous": 0, "steps": 1}.get(engine)
        if mode is None:
            raise ValueError(f"unknown serving engine {engine!r}")
        cfg = _Config(max_step_code_blocks, steps_in_flight, harq_bytes, staging_bytes, iterations, offset_beta,
                      scale, app_clamp, latency_steps, backlog_code_blocks, code, mode, idle_us)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_serve_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h.value
        self._keep = {}

    def set_tiles(self, tiles):
        """Work-item sizes per shape, {(bg, z): codewords} (autotune.tune_tiles)."""
        arr = np.ascontiguousarray(np.asarray([(bg, z, t) for (bg, z), t in tiles.items()], dtype=np.int32)
                                   .reshape(-1, 3))
        _lib.check(_lib.load().syndrome_serve_set_tiles(self._h, arr.ctypes.data if len(arr) else None, len(arr)))

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            _lib.load().syndrome_serve_destroy(h)
        self._keep = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, tb_id, tb_size, target_rate, qm, g, rv, llr):
        """Queues one transmission.  llr: C * E f32 LLRs as a numpy array (host) or a
        CUDA tensor; it is kept alive until the transmission's result is polled."""
        try:
            import torch
            on_dev = isinstance(llr, torch.Tensor) and llr.is_cuda
        except ImportError:
            on_dev = False
        if on_dev:
            if llr.dtype != torch.float32 or not llr.is_contiguous():
                raise TypeError("llr must be a contiguous float32 tensor")
            ptr, n = llr.data_ptr(), llr.numel()
        else:
            llr = np.ascontiguousarray(llr, dtype=np.float32)
            ptr, n = llr.ctypes.data, llr.size
        _lib.check(_lib.load().syndrome_serve_submit(self._h, tb_id, tb_size, target_rate, qm, g, rv,
                                                     ctypes.c_void_p(ptr), n, int(on_dev)))
        self._keep.setdefault(tb_id, []).append(llr)

    def poll(self, timeout_us=0, cap=1024):
        """Completed transmissions: dicts with the DecodeReport fields and latency_us."""
        buf = (_Result * cap)()
        n = ctypes.c_size_t(0)
        _lib.check(_lib.load().syndrome_serve_poll(self._h, buf, cap, ctypes.byref(n), int(timeout_us)))
        out = []
        for r in buf[: n.value]:
            keep = self._keep.get(r.tb_id)
            if keep:
                keep.pop(0)
                if not keep:
                    del self._keep[r.tb_id]
            cb = [bool((r.cb_crc[i // 32] >> (i % 32)) & 1) for i in range(r.num_code_blocks)]
            out.append(dict(tb_id=r.tb_id, crc_ok=bool(r.crc_ok), max_iters_used=r.max_iters_used,
                            harq_tx_count=r.harq_tx_count, cb_crc=cb, latency_us=r.latency_us))
        return out

    def wait(self, count, timeout_s=60.0):
        """Polls until `count` results arrived (raises TimeoutError otherwise)."""
        import time

        out, t_end = [], time.time() + timeout_s
        while len(out) < count:
            if time.time() > t_end:
                raise TimeoutError(f"{len(out)} of {count} results after {timeout_s} s")
            out += self.poll(timeout_us=20000)
        return out

    def fetch(self, tb_id, tb_size):
        bits = np.zeros(tb_size, dtype=np.uint8)
        _lib.check(_lib.load().syndrome_serve_fetch(self._h, tb_id, bits.ctypes.data, tb_size))
        return bits

    def release(self, tb_id):
        _lib.check(_lib.load().syndrome_serve_release(self._h, tb_id))

    def stats(self):
        v = np.zeros(14, dtype=np.int64)
        _lib.check(_lib.load().syndrome_serve_stats(self._h, v.ctypes.data))
        keys = ("steps", "code_blocks", "transmissions", "harq_bytes_used", "pending", "in_flight", "tbs_held",
                "max_pending", "items", "item_threads", "decode_us", "step_us", "host_launch_us", "host_finish_us")
        return dict(zip(keys, (int(x) for x in v)))

    def core_stats(self):
        """Continuous engine: items the persistent kernel finished, microseconds its CTAs
        spent (busy, combine, decode, crc, finish) and the worker's iterations and
        microseconds (admit, publish, complete).  Zeros for the step engine."""
        v = np.zeros(10, dtype=np.float64)
        _lib.check(_lib.load().syndrome_serve_core_stats(self._h, v.ctypes.data))
        keys = ("items", "busy_us", "combine_us", "decode_us", "crc_us", "finish_us", "loops", "admit_us",
                "publish_us", "complete_us")
        return dict(zip(keys, (float(x) for x in v)))

    def run_load(self, pool, offered_tb_per_s, duration_s, max_transmissions=4, seed=0, latencies=False):
        """Open-loop Poisson load (syndrome_serve_run_load).  pool: list of dicts with
        tb_size, target_rate, qm, g and llrs = four contiguous float32 CUDA tensors (the
        transmissions with RV 0, 2, 3, 1).  Returns the report as a dict (plus the
        per-block latencies in arrival order when latencies=True)."""
        arr = (_LoadTb * len(pool))()
        for i, p in enumerate(pool):
            arr[i].tb_size, arr[i].target_rate, arr[i].qm, arr[i].g = p["tb_size"], p["target_rate"], p["qm"], p["g"]
            for k in range(4):
                t = p["llrs"][k]
                if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
                    raise TypeError("pool LLRs must be contiguous float32 CUDA tensors")
                arr[i].llr[k] = t.data_ptr()
            arr[i].llr_len = p["llrs"][0].numel()
        spec = _LoadSpec(offered_tb_per_s, duration_s, max_transmissions, seed)
        rep = _LoadReport()
        cap = int(offered_tb_per_s * duration_s * 2 + 1024) if latencies else 0
        lat = np.zeros(cap, dtype=np.float64)
        _lib.check(_lib.load().syndrome_serve_run_load(self._h, arr, len(pool), ctypes.byref(spec), ctypes.byref(rep),
                                                       lat.ctypes.data if cap else None, cap))
        out = {k: getattr(rep, k) for k, _ in _LoadReport._fields_}
        if latencies:
            out["latencies_us"] = lat[: rep.tbs]
        return out

