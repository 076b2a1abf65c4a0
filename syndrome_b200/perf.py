"""Throughput of one batched decode shape on the GPU, as decoded information Gbit/s.

    python -m syndrome_b200.perf --code wifi --z 81 --rate 1/2 --precision f32 --count 32768
    python -m syndrome_b200.perf --code nr --bg 0 --z 384 --precision f32 --count 4096

Seeded random codewords (GPU encoder) sent as BPSK over AWGN at --ebno dB; 5G NR
codewords drop their first 2Z bits (punctured) and decode with the 5G prologue.  The
LLRs are device-resident; the timed region is --repeats back-to-back decodes with
packed hard decisions and iteration counts out, between CUDA events on the current
stream, after one warm-up decode.  Prints one JSON line.
"""
import argparse
import json


def make_llrs(args):
    """(decoder, llr tensor, info bits K, llr_offset, nr prologue) for the requested shape."""
    import torch

    from .qc_ldpc import QcLdpcDecoder, QcLdpcEncoder, wifi_ldpc_decoder, wifi_ldpc_encoder

    gen = torch.Generator(device="cuda")
    gen.manual_seed(args.seed)
    if args.code == "nr":
        dec = QcLdpcDecoder.with_lifting_size(args.bg, args.z, args.beta)
        enc = QcLdpcEncoder.new(args.bg, args.z)
        skip = 2 * args.z
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
    return dec, llr, k, skip, args.code == "nr"


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
    args = p.parse_args(argv)

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
