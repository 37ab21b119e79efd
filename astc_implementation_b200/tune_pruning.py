"""Speed and quality of proposal-search settings against the full search.

    python -m astc_implementation_b200.tune_pruning --size 1024 --footprints 4,6 \\
        --settings '[{"max_partitionings": 4, "block_modes": 16, "refine_candidates": 2}]'

Encodes synthetic textures (generator seeds 7-10, not used for training) with the full search
and with each setting (unspecified fields take the ASTCEncoder.set_pruning defaults), and prints
one JSON line per run: device milliseconds per texture, speed-up, PSNR delta per texture,
routes, and the per-launch milliseconds of the last encode.  Needs a GPU.
"""
import argparse
import json

import numpy as np

from . import ASTCEncoder, decode, psnr
from . import proposal, synth


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--footprints", default="4,6", help="square footprints, comma separated")
    ap.add_argument("--seeds", default="7,8,9,10")
    ap.add_argument("--settings", default="[{}]", help="JSON list of set_pruning keyword sets")
    args = ap.parse_args()
    side = args.size
    seeds = [int(v) for v in args.seeds.split(",")]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    for bx in (int(v) for v in args.footprints.split(",")):
        imgs = [synth.make_texture(side, side, s) for s in seeds]
        enc = ASTCEncoder(device=0, stage_timing=True)
        enc.secondaryInit(side, side, bx, bx)
        d_in = [torch.from_numpy(im.reshape(-1)).cuda() for im in imgs]
        out = torch.empty(enc.numBlocks * 16, dtype=torch.uint8, device="cuda")

        def timed():
            enc.encode_device(d_in[0].data_ptr(), out.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for d in d_in:
                enc.encode_device(d.data_ptr(), out.data_ptr(), stream.cuda_stream)
            t1.record(stream)
            torch.cuda.synchronize()
            det, _ = enc.stage_times_detail()
            return t0.elapsed_time(t1) / len(d_in), [round(float(x), 3) for x in det]

        def quality():
            return [psnr(decode(bx, bx, side, side, enc.encode(im)), im) for im in imgs]

        ms_full, det = timed()
        q_full = quality()
        print(json.dumps({"footprint": bx, "method": "full", "ms": round(ms_full, 3), "psnr": [round(q, 3) for q in q_full],
                          "launch_ms": det}), flush=True)
        enc.set_proposal_net(proposal.load_weights(bx, bx))
        for st in json.loads(args.settings):
            enc.set_pruning(True, **st)
            ms, det = timed()
            q = quality()
            d = [a - b for a, b in zip(q, q_full)]
            print(json.dumps({"footprint": bx, "method": st, "ms": round(ms, 3), "speedup": round(ms_full / ms, 3),
                              "dpsnr_mean": round(float(np.mean(d)), 3), "dpsnr": [round(x, 3) for x in d],
                              "routes": enc.pruning_stats(), "launch_ms": det}), flush=True)
        enc.close()


if __name__ == "__main__":
    main()
