"""Times the reference's own CPU solvers on this host (measurement
infrastructure; the product never calls it).

``parallel_n_queens`` and ``serial_n_queens`` (src/n_queens.cpp:115-163) run
unchanged from ``oracle/_ref/libnq_ref.so`` (the reference's n_queens.cpp
compiled from its sources by oracle/Makefile).  ``parallel_n_queens`` forces
32 OpenMP threads with static scheduling (src/n_queens.cpp:152-153) whatever
the core count; the JSON line records the host's core count and CPU model
beside the time.

    python -m oracle.time_reference_cpu --N 20 --k 6 [--serial]
"""
from __future__ import annotations

import argparse
import json
import os
import time

from . import ref, ref_available

# Published totals (README.md:16-25) to check the result against.
PUBLISHED = {13: 73712, 14: 365596, 15: 2279184, 16: 14772512, 17: 95815104, 18: 666090624, 19: 4968057848,
             20: 39029188884, 21: 314666222712, 22: 2691008701644}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, required=True)
    ap.add_argument("--k", type=int, required=True)
    ap.add_argument("--serial", action="store_true", help="serial_n_queens instead of parallel_n_queens")
    args = ap.parse_args()
    if not ref_available():
        raise SystemExit("oracle/_ref/libnq_ref.so is not built: make -C oracle REF_SRC=<reference>/src")
    L = ref()
    fn = L.nqref_serial if args.serial else L.nqref_parallel
    t = time.perf_counter()
    total = int(fn(args.N, args.k))
    dt = time.perf_counter() - t
    print(json.dumps({"solver": "serial_n_queens" if args.serial else "parallel_n_queens",
                      "N": args.N, "k": args.k, "total": total,
                      "total_ok": PUBLISHED.get(args.N) in (None, total), "seconds": dt,
                      "omp_threads": 1 if args.serial else 32, "host_cores": os.cpu_count(),
                      "cpu_model": cpu_model()}), flush=True)


if __name__ == "__main__":
    main()
