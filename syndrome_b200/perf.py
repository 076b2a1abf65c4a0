"""Throughput of one batched decode shape on the GPU, as decoded information Gbit/s.

    python -m syndrome_b200.perf --code wifi --z 81 --rate 1/2 --precision f32 --count 32768
    python -m syndrome_b200.perf --code nr --bg 0 --z 384 --precision f32 --count 4096
    python -m syndrome_b200.perf --pipeline --code nr --bg 0 --z 384 --iterations 5 --ebno 2.0

Seeded random codewords (GPU encoder) sent as BPSK over AWGN at --ebno dB; 5G NR
codewords drop their first 2Z bits (punctured) and decode with the 5G prologue.  The
LLRs are device-resident; the timed region is --repeats back-to-back decodes with
packed hard decisions and iteration counts out, between CUDA events on the current
stream, after one warm-up decode.  Prints one JSON line.

--pipeline instead drives the LdpcPipeline frame API (ldpc_pipeline.rs: acquire, fill
the frame's N f32 LLRs from host memory, submit, try_recv, release) with --count
frames after --count / 8 warm-up frames, every bit of the codeword sent (as the
reference's pipeline benchmark), timed by the host clock.  It reports frames/s,
decoded information Gbit/s and Melem/s = N x iterations used / t (the reference's
pipeline unit).
"""
import argparse
import json


def make_llrs(args, puncture=True):
    """(decoder, llr tensor, info bits K, llr_offset, nr prologue) for the requested shape;
    puncture=False sends every bit of a 5G NR codeword (no 2Z puncturing, no prologue)."""
    import torch

    from .qc_ldpc import QcLdpcDecoder, QcLdpcEncoder, wifi_ldpc_decoder, wifi_ldpc_encoder

    gen = torch.Generator(device="cuda")
    gen.manual_seed(args.seed)
    if args.code == "nr":
        dec = QcLdpcDecoder.with_lifting_size(args.bg, args.z, args.beta)
        enc = QcLdpcEncoder.new(args.bg, args.z)
        skip = 2 * args.z if puncture else 0
    else:
        rn, rd = (int(x) for x in args.rate.split("/"))
        dec = wifi_ldpc_decoder(args.z, rn, rd, args.beta)
        enc = wifi_ldpc_encoder(args.z, rn, rd)
        skip = 0
    n, k = dec.variable_node_count(), enc.info_bit_count()
    info = torch.randint(0, 2, (args.count, k), generator=gen, device="cuda", dtype=torch.uint8)
    cw = enc.encode_batch_device(info)
    rate = k / (n - skip)
    sigma = (1.0 / (2.0 * rate * 10.0 ** (args.ebno / 10.0))) ** 0.5
    x = 1.0 - 2.0 * cw[:, skip:].float()
    llr = (2.0 * (x + sigma * torch.randn(x.shape, generator=gen, device="cuda")) / sigma ** 2).contiguous()
    if args.precision == "int8":
        llr = torch.clamp(torch.round(llr * args.scale), -127, 127).to(torch.int8).contiguous()
    return dec, llr, k, skip, args.code == "nr" and puncture


def run_pipeline(args):
    """Frames through LdpcPipeline as fast as the host loop submits them (see --pipeline)."""
    import time

    import numpy as np

    from .ldpc_pipeline import LdpcPipeline

    gen_args = argparse.Namespace(**dict(vars(args), precision="f32", count=min(args.count, 256)))
    dec, llr, k, _, _ = make_llrs(gen_args, puncture=False)
    src = llr.cpu().numpy().astype(np.float32)
    n = dec.variable_node_count()
    pipe = (LdpcPipeline.with_workers(dec, args.iterations, args.workers) if args.workers
            else LdpcPipeline.new(dec, args.iterations))

    def drive(count):
        done = iters = sent = 0
        while done < count:
            progressed = False
            if sent < count:
                f = pipe.acquire()
                if f is not None:
                    np.copyto(f.llr_mut(), src[sent % src.shape[0]])
                    pipe.submit(f)
                    sent += 1
                    progressed = True
            g = pipe.try_recv()
            if g is not None:
                iters += g.iterations_used()
                pipe.release(g)
                done += 1
                progressed = True
            if not progressed:
                time.sleep(0)
        return iters

    drive(max(args.count // 8, 16))
    t0 = time.perf_counter()
    iters = drive(args.count)
    t = time.perf_counter() - t0
    print(json.dumps(dict(api="LdpcPipeline", code=args.code, z=args.z, bg=args.bg, precision="f32",
                          frames=args.count, workers=pipe.worker_count(), iterations_max=args.iterations,
                          ebno_db=args.ebno, seconds=round(t, 4), frames_per_s=round(args.count / t, 1),
                          gbps=round(args.count * k / t / 1e9, 3), melem_per_s=round(n * iters / t / 1e6, 1),
                          mean_iterations=round(iters / args.count, 3))))


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--code", choices=["nr", "wifi"], default="nr")
    p.add_argument("--bg", type=int, default=0, help="5G NR base graph: 0 = BG1, 1 = BG2")
    p.add_argument("--z", type=int, default=384)
    p.add_argument("--rate", default="1/2", help="802.11 code rate")
    p.add_argument("--precision", choices=["int8", "f32"], default="int8")
    p.add_argument("--kernel", default="auto", choices=["auto", "generic", "generic_global", "nr", "pair"])
    p.add_argument("--count", type=int, default=4096)
    p.add_argument("--iterations", type=int, default=8)
    p.add_argument("--ebno", type=float, default=1.5)
    p.add_argument("--beta", type=float, default=0.5)
    p.add_argument("--scale", type=float, default=8.0)
    p.add_argument("--repeats", type=int, default=5)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--pipeline", action="store_true", help="drive the LdpcPipeline frame API instead")
    p.add_argument("--workers", type=int, default=0, help="pipeline worker threads (0: the default)")
    args = p.parse_args(argv)
    if args.pipeline:
        run_pipeline(args)
        return

    import torch

    from .autotune import _time_ms
    from .qc_ldpc import QuantParams

    dec, llr, k, skip, nr = make_llrs(args)
    dec.set_kernel(args.kernel)
    out = {"hard_packed": torch.empty((args.count, (k + 31) // 32), dtype=torch.int32, device="cuda"),
           "iters": torch.empty((args.count,), dtype=torch.int32, device="cuda")}
    kw = dict(llr_offset=skip, nr_prologue=nr, hard_bits=k, out=out)
    if args.precision == "int8":
        quant = QuantParams()
        run = lambda: dec.decode_batch_i8(llr, args.iterations, quant=quant, **kw)  # noqa: E731
    else:
        run = lambda: dec.decode_batch_f32(llr, args.iterations, **kw)  # noqa: E731
    ms = _time_ms(run, args.repeats)
    shape = {"code": args.code, "z": args.z, "precision": args.precision, "kernel": args.kernel,
             "count": args.count, "iterations_max": args.iterations, "ebno_db": args.ebno}
    shape.update({"bg": args.bg} if nr else {"rate": args.rate})
    print(json.dumps(dict(shape, ms=round(ms, 4), gbps=round(args.count * k / ms / 1e6, 3),
                          mean_iterations=round(float(out["iters"].float().mean()), 3))))


if __name__ == "__main__":
    main()
