#!/usr/bin/env python3
"""Autotunes the pass plans of this device and writes them to a plan file.

    python era-boojum-cuda_b200/tune_plans.py [--out era-boojum-cuda_b200/plans_b200.txt]

For every log_n in 12..23 and blowup in {1 (plain NTT), 2, 4, 8} it times all
candidate window splits and then the launch knobs of the best one (bc_autotune)
on 2^27 input elements of columns (2^28 output elements at most) and keeps the
fastest; bc_ntt.load_tuned_plans() loads the file into a process.
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main():
    import torch

    import bc_ntt

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "plans_b200.txt"))
    ap.add_argument("--log-n", type=int, nargs=2, default=(12, 23))
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    bc_ntt.Context.create()
    bc_ntt.plan_table_clear()
    lines = []
    for log_n in range(args.log_n[0], args.log_n[1] + 1):
        for log_b in (0, 1, 2, 3):
            cols = max(1, (1 << 27) >> (log_n + max(0, log_b - 1)))
            rep = bc_ntt.autotune(log_n, log_b, cols, args.reps)
            best = rep.strip().splitlines()[-1]
            lines.append(f"# log_n {log_n} blowup {1 << log_b} cols {cols}: " + " | ".join(rep.strip().splitlines()))
            print(f"log_n={log_n} blowup={1 << log_b}: {best}", flush=True)
    name = torch.cuda.get_device_name(0)
    with open(args.out, "w") as f:
        f.write(f"# pass plans tuned on {name} by tune_plans.py; format: log_n log_blowup npasses (K C)... "
                "[k walk top_walk top_mode top_dbuf occ]\n")
        for line in lines:
            f.write(line + "\n")
        f.write(bc_ntt.plan_table_export())
    print("wrote", args.out)


if __name__ == "__main__":
    main()
