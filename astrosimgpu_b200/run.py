"""Run a shipped (or given) network configuration on the B200 engine, with
checkpoint and resume.

    python -m astrosimgpu_b200.run --config paper_sparse_dt005 --steps 16000 --save ck.bin
    python -m astrosimgpu_b200.run --config paper_sparse_dt005 --load ck.bin --steps 8 --plain
    python -m astrosimgpu_b200.run --serving 1000000 --steps 120 --plain

A checkpoint is the engine's device state of one network (asg_checkpoint):
resuming it in a network built from the same configuration continues the
run bit for bit.  `--plain` launches one kernel per step without CUDA graphs
(each launch then shows up on its own in a profiler).  `--serving N` runs the
serving-shaped network of N neurons and N astrocytes instead (use_case
parameters, fixed in-degree 100, generated on the device), the shape of the
largest request of the serving stream.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

from . import _lib
from .network import Model, Network, config_path


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--config", default="paper_sparse_dt005",
                    help="shipped configuration name or path to a JSON file")
    ap.add_argument("--serving", type=int, default=0,
                    help="run the serving-shaped network of this many neurons instead")
    ap.add_argument("--seed", type=int, default=99, help="seed of the --serving network")
    ap.add_argument("--steps", type=int, required=True)
    ap.add_argument("--save", help="write a checkpoint after the steps")
    ap.add_argument("--load", help="resume from a checkpoint before the steps")
    ap.add_argument("--plain", action="store_true", help="one launch per step, no graphs")
    ap.add_argument("--chunk", type=int, default=0,
                    help="steps per chunk (0: the engine's default for the network size)")
    args = ap.parse_args(argv)

    if args.serving:
        from .workloads import serving_config
        model = Model(text=serving_config(args.serving, args.seed, 100.0), pre_time=0.0,
                      fixed_indegree=100, gen_device=0)
        args.config = f"serving {args.serving} neurons, seed {args.seed}"
    else:
        path = args.config if os.path.exists(args.config) else config_path(args.config)
        model = Model(path, pre_time=0.0)
    opts = dict(chunk_steps=args.chunk)
    if args.plain:
        opts["use_graphs"] = -1
    net = Network(model, record=_lib.RecordOpts(0, 10, 1, 0, 0), **opts)
    if args.load:
        with open(args.load, "rb") as f:
            net.restore(f.read())
    first = net.current_step
    t0 = time.perf_counter()
    net.step(args.steps)
    wall = time.perf_counter() - t0
    ms, kernels = net.last_timing()
    if args.save:
        with open(args.save, "wb") as f:
            f.write(net.checkpoint())
    print(json.dumps({"config": args.config, "from_step": first, "steps": args.steps,
                      "device_ms": ms, "kernels": kernels, "wall_s": wall,
                      "counters": net.counters()}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
