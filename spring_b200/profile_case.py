"""One small case of one path, for a profiler (ncu) or a quick timing: the synthetic rocksalt cell
at a given mesh, one call of the chosen entry point, its kernel times printed.

    python -m spring_b200.profile_case v4 --mesh 8 --q0 3 [--precision bf16x3]
    python -m spring_b200.profile_case v3 --mesh 16 [--precision bf16x3]
    python -m spring_b200.profile_case bte --mesh 12
    python -m spring_b200.profile_case v3 --mesh 24 --temps 100,300,700 --warm 30 --repeat 10 --profiled 10
"""
from __future__ import annotations

import argparse
import time

SIGMA = 0.3767  # 2 cm^-1 in rad/ps


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["v3", "v4", "bte"])
    ap.add_argument("--mesh", type=int, default=8)
    ap.add_argument("--q0", type=int, default=0, help="irreducible points (0: all)")
    ap.add_argument("--precision", default="bf16x3", choices=["fp64", "bf16", "bf16x3"])
    ap.add_argument("--repeat", type=int, default=2, help="calls")
    ap.add_argument("--warm", type=int, default=0,
                    help="extra calls before them: a few cold calls run below full clocks, so use ~30 for timings")
    ap.add_argument("--profiled", type=int, default=1, help="the last this many calls are profiled (per-call means)")
    ap.add_argument("--temps", default="300", help="temperatures in K, comma-separated")
    a = ap.parse_args()
    from . import synthetic as S
    from .api import from_crystal
    cr = S.build("rocksalt2", fc4=a.case == "v4")
    temps = [float(x) for x in a.temps.split(",")]
    ctx, _ = from_crystal(cr, (a.mesh,) * 3, temps, with_fc4=a.case == "v4")
    ctx.set_precision(a.precision)
    n = ctx.nq0 if a.q0 <= 0 else min(a.q0, ctx.nq0)
    calls = a.warm + a.repeat
    prof = max(1, min(a.profiled, calls))
    for r in range(calls):
        if r == calls - prof:
            ctx.set_profiling(True)
        t = time.time()
        if a.case == "v3":
            ctx.reset_linewidths()
            ctx.linewidth3(1, n, "gauss", SIGMA, want=False)
        elif a.case == "v4":
            ctx.linewidth4(1, n, "gauss", SIGMA)
        else:
            ctx.kappa_iter_gauss(SIGMA, eps_k=1e-6)
        ctx.synchronize()
        wall = time.time() - t
    total_ms, total_n = ctx.kernel_time("")
    names = {"v3": ("k_v3tc<", "k_v3s", "k_tc_"), "v4": ("k_v4tc", "k4_", "k_enum4"),
             "bte": ("k_v3s", "k_bteg_", "k_bte_")}[a.case]
    print(f"{a.case} mesh {a.mesh}^3, {n} q0, {len(temps)} T, {a.precision}: last call wall {wall * 1e3:.1f} ms, "
          f"{total_n} profiled launches over {prof} call(s), {total_ms / prof:.3f} ms per call")
    for k in names:
        ms, cnt = ctx.kernel_time(k)
        print(f"  {k:14s} {ms / prof:10.4f} ms per call  {cnt} launches")
    ctx.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
