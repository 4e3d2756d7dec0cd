"""Profiling and report tooling: GPU time per kernel, result tables.

The reference's ``tools/kernel_breakdown.py`` (GPU time per kernel category
from an Nsight Systems export) and ``tools/summary.py`` (results table) work
on nsys captures. Here the sources are the plan's own CUDA-event phase ring
(``lrd_plan_set_profiling`` / ``lrd_plan_phase_ms``), an ``ncu`` launch list
(``--metrics gpu__time_duration.sum --csv``) and ``bench.py``'s JSON lines.

    python -m lowrank_gpu_fastest_b200.report breakdown [--shape 96,96,48,48] [--form plain]
    python -m lowrank_gpu_fastest_b200.report target [--shape ...] [--form ...] [--reps 2]
    python -m lowrank_gpu_fastest_b200.report ncu-table launches.csv [--skip REGEX]
    python -m lowrank_gpu_fastest_b200.report summary bench1.json [bench2.json ...]
    python -m lowrank_gpu_fastest_b200.report rank-agreement case1.npz [case2.npz ...] [--forms plain,accurate]
    python -m lowrank_gpu_fastest_b200.report harness [--shape ...] [--form ...] [--phantom ladder|lowrank]
                                                      [--ref step0_out.npy] [--json out.json]

``harness`` times the library's host->host ``denoise`` the way the ladder's
``common.run`` (common.py:103-172) times a rung: warm-up call, best of up to
5 calls within 60 s, relative L2 against a saved step-0 output when given.

``target`` is the workload for an ncu capture: it denoises the synthetic
volume ``reps`` times (device-resident) and exits.
"""

from __future__ import annotations

import argparse
import csv
import json
import re
import statistics
import sys

PHASE_LABELS = {"center": "centre (temporal mean)", "gram": "Gram (column, TMA-staged)",
                "eigh_mp": "eigensolve + MP rank + refine", "recon": "reconstruction + overlap-add"}


def _shape(s):
    return tuple(int(v) for v in s.split(","))


def phase_breakdown(shape=(96, 96, 48, 48), patch=(11, 11, 11), stride=3, form="plain", reps=10, seed=0):
    """Device ms per phase (mean over ``reps`` calls), plus the host-buffer
    call's H2D / D2H copies timed alone with CUDA events."""
    import numpy as np
    import torch

    from . import api
    from .harness import make_phantom_lowrank

    vol = make_phantom_lowrank(shape, seed=seed)[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    d = torch.from_numpy(vol).to(dev)
    out = torch.empty_like(d)
    plan = api.get_plan(shape, patch, stride, form=form)
    for _ in range(3):
        api.denoise(d, patch, stride, form=form, out=out)
    torch.cuda.synchronize()
    plan.set_profiling(True)
    for _ in range(reps):
        api.denoise(d, patch, stride, form=form, out=out)
    torch.cuda.synchronize()
    ms, n = plan.phase_ms()
    plan.set_profiling(False)
    ms = {k: v / max(n, 1) for k, v in ms.items()}
    h = torch.from_numpy(vol).pin_memory()
    ho = torch.empty_like(h).pin_memory()
    s, e, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    copies = []
    for _ in range(reps):
        s.record()
        d.copy_(h, non_blocking=True)
        e.record()
        ho.copy_(out, non_blocking=True)
        e2.record()
        torch.cuda.synchronize()
        copies.append((s.elapsed_time(e), e.elapsed_time(e2)))
    ms["memcpy H2D"] = statistics.mean(c[0] for c in copies)
    ms["memcpy D2H"] = statistics.mean(c[1] for c in copies)
    n_p = plan.n_patches
    return dict(shape=list(shape), patch=list(patch), stride=stride, form=form, patches=n_p,
                ms=ms, kernels_ms=sum(v for k, v in ms.items() if not k.startswith("memcpy")),
                volume_mib=float(np.prod(shape)) * 4 / 2**20)


def kernel_name(raw):
    """Short kernel name from an ncu 'Kernel Name' cell (drops namespaces,
    parameter lists and template arguments)."""
    n = re.sub(r"\(anonymous namespace\)", "anon", raw)
    n = n.split("(")[0]
    n = re.sub(r"^void\s+", "", n)
    depth, cut = 0, ""
    for ch in n:  # drop template arguments
        if ch == "<":
            depth += 1
        elif ch == ">":
            depth -= 1
        elif depth == 0:
            cut += ch
    return cut.split("::")[-1] or raw[:40]


def ncu_launch_table(path, skip=None):
    """Per kernel: launches, total ms, share of the listed time (ncu launch
    list CSV with gpu__time_duration.sum). ``skip``: regex of kernel names to
    leave out (e.g. a library GEMM a benchmark runs for its own reference)."""
    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hi]
    ki, mi, vi, ui = (h.index(c) for c in ("Kernel Name", "Metric Name", "Metric Value", "Metric Unit"))
    scale = {"ns": 1e-6, "usecond": 1e-3, "us": 1e-3, "ms": 1.0, "msecond": 1.0, "nsecond": 1e-6}
    agg = {}
    for r in rows[hi + 1:]:
        if len(r) <= vi or r[mi] != "gpu__time_duration.sum":
            continue
        k = kernel_name(r[ki])
        if skip and (re.search(skip, k) or re.search(skip, r[ki])):
            continue
        v = float(r[vi].replace(",", "")) * scale.get(r[ui], 1e-6)
        a = agg.setdefault(k, [0, 0.0])
        a[0] += 1
        a[1] += v
    total = sum(a[1] for a in agg.values()) or 1.0
    return [dict(kernel=k, launches=n, total_ms=t, mean_us=1e3 * t / n, share=t / total)
            for k, (n, t) in sorted(agg.items(), key=lambda kv: -kv[1][1])]


def markdown_table(header, rows):
    out = ["| " + " | ".join(header) + " |", "|" + "---|" * len(header)]
    out += ["| " + " | ".join(str(c) for c in r) + " |" for r in rows]
    return "\n".join(out)


def summary(lines):
    """Markdown table of bench.py JSON lines."""
    rows = []
    for d in lines:
        cfg = d.get("config", {})
        wl = cfg.get("workload", d.get("workload", ""))
        e2e = d.get("e2e") or {}
        roof = d.get("roofline") or {}
        rows.append([d.get("impl", "ours"), wl, cfg.get("form", ""), d.get("n_gpus", 1),
                     f"{d['value']:,.0f} {d['unit']}", f"{d.get('ms_per_step', float('nan')):.3f}",
                     f"{e2e['value']:,.0f}" if "value" in e2e else "",
                     f"{roof.get('kernel', '')} {roof.get('frac', 0):.3f}" if roof else "",
                     (d.get("clocks") or {}).get("sm_mhz", "")])
    return markdown_table(["impl", "workload", "form", "GPUs", "value", "ms/step", "e2e", "roofline frac",
                           "SM MHz"], rows)


def regenerate_input(rec):
    """Input volume of a case record (``gen``: "ref" = the ladder's phantom,
    "lowrank" = the benchmark phantom, "const" = a constant 3.0 volume;
    ``shape``; ``gen_kwargs`` as a Python literal)."""
    import ast

    import numpy as np

    from .harness import make_phantom, make_phantom_lowrank

    shape = tuple(int(s) for s in rec["shape"])
    kw = ast.literal_eval(str(rec["gen_kwargs"]))
    gen = str(rec["gen"])
    if gen == "ref":
        return make_phantom(shape, **kw)[0]
    if gen == "lowrank":
        return make_phantom_lowrank(shape, **kw)[0]
    if gen == "const":
        return np.full(shape, 3.0, dtype=np.float32)
    raise ValueError(f"unknown generator {gen!r}")


def count_mismatches(ranks, ranks32, ranks64):
    """MP-rank disagreements of ``ranks`` with a float32 and a float64 run of
    the step-0 loop, and of those two runs with each other."""
    import numpy as np

    r, a, b = (np.asarray(v).astype(np.int64) for v in (ranks, ranks32, ranks64))
    return dict(n=int(len(r)), vs_step0=int((r != a).sum()), vs_fp64=int((r != b).sum()),
                step0_vs_fp64=int((a != b).sum()))


def rank_agreement(paths, forms=("plain", "accurate", "tensor", "tensor_bf16")):
    """Rank agreement in the manner of the ladder's micro/rank_agreement.py:
    46-102 (which counts the MP-rank mismatches of FP32 routes against an FP64
    SVD): for every case file (an ``.npz`` with the input's generator, shape,
    patch, stride and the per-patch ranks of step 0 run in float32,
    ``ranks``, and in float64, ``ranks64``) and every form, the library's
    ranks (device-resident call) against both. Returns a list of rows."""
    import os

    import numpy as np
    import torch

    from . import api

    rows = []
    for path in paths:
        d = np.load(path)
        vol = regenerate_input(d)
        patch, stride = tuple(int(v) for v in d["patch"]), int(d["stride"])
        dv = torch.from_numpy(vol).cuda()
        for form in forms:
            _, rk = api.denoise(dv, patch, stride, form=form, return_ranks=True)
            rk = rk.cpu().numpy()
            rows.append(dict(case=os.path.basename(path).rsplit(".", 1)[0], shape=tuple(vol.shape),
                             patch=patch, stride=stride, form=form,
                             **count_mismatches(rk, d["ranks"], d["ranks64"])))
        del dv
    return rows


def rank_table(rows):
    return markdown_table(["case", "shape", "patch / stride", "form", "patches", "vs step 0 (fp32)",
                           "vs fp64", "step 0 vs fp64"],
                          [[r["case"], "x".join(map(str, r["shape"])), f"{r['patch'][0]}^3 / {r['stride']}"
                            if len(set(r["patch"])) == 1 else f"{r['patch']} / {r['stride']}", r["form"], r["n"],
                            r["vs_step0"], r["vs_fp64"], r["step0_vs_fp64"]] for r in rows])


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m lowrank_gpu_fastest_b200.report")
    sub = ap.add_subparsers(dest="cmd", required=True)
    for name in ("breakdown", "target"):
        p = sub.add_parser(name)
        p.add_argument("--shape", type=_shape, default=(96, 96, 48, 48))
        p.add_argument("--patch", type=_shape, default=(11, 11, 11))
        p.add_argument("--stride", type=int, default=3)
        p.add_argument("--form", default="plain")
        p.add_argument("--reps", type=int, default=10 if name == "breakdown" else 2)
    p = sub.add_parser("ncu-table")
    p.add_argument("csv")
    p.add_argument("--skip", default=None)
    p = sub.add_parser("summary")
    p.add_argument("files", nargs="+")
    p = sub.add_parser("harness")
    p.add_argument("--shape", type=_shape, default=(96, 96, 48, 48))
    p.add_argument("--patch", type=_shape, default=(11, 11, 11))
    p.add_argument("--stride", type=int, default=3)
    p.add_argument("--form", default="plain")
    p.add_argument("--phantom", choices=["ladder", "lowrank"], default="ladder")
    p.add_argument("--repeats", type=int, default=5)
    p.add_argument("--ref", default=None, help=".npy of the step-0 output on the same phantom")
    p.add_argument("--json", default=None)
    p = sub.add_parser("rank-agreement")
    p.add_argument("cases", nargs="+")
    p.add_argument("--forms", default="plain,accurate,tensor,tensor_bf16")
    a = ap.parse_args(argv)
    if a.cmd == "breakdown":
        r = phase_breakdown(a.shape, a.patch, a.stride, a.form, a.reps)
        print(f"volume {tuple(r['shape'])}, patch {tuple(r['patch'])}, stride {r['stride']}, "
              f"{r['patches']} patches, form {r['form']}\n")
        print(markdown_table(["GPU time (ms)", "mean"],
                             [[PHASE_LABELS.get(k, k), f"{v:.3f}"] for k, v in r["ms"].items()]
                             + [["*kernels total*", f"*{r['kernels_ms']:.3f}*"]]))
        print(json.dumps(r))
    elif a.cmd == "target":
        import torch

        from . import api
        from .harness import make_phantom_lowrank

        vol = make_phantom_lowrank(a.shape)[0]
        d = torch.from_numpy(vol).cuda()
        out = torch.empty_like(d)
        for _ in range(a.reps):
            api.denoise(d, a.patch, a.stride, form=a.form, out=out)
        torch.cuda.synchronize()
        print("ok", float(out.mean()))
    elif a.cmd == "ncu-table":
        t = ncu_launch_table(a.csv, a.skip)
        print(markdown_table(["kernel", "launches", "total ms", "mean us", "share"],
                             [[r["kernel"], r["launches"], f"{r['total_ms']:.3f}", f"{r['mean_us']:.1f}",
                               f"{100 * r['share']:.1f}%"] for r in t]))
    elif a.cmd == "harness":
        import functools

        import numpy as np
        import torch

        from . import api
        from .harness import make_phantom, make_phantom_lowrank, run
        from .problem import n_patches

        gen = make_phantom if a.phantom == "ladder" else make_phantom_lowrank
        noisy, clean = gen(a.shape)
        ref = np.load(a.ref) if a.ref else None
        fn = functools.partial(api.denoise, patch=a.patch, stride=a.stride, form=a.form)
        res, _ = run(f"lrd_{a.form}", fn, noisy, clean, ref, n_patches(a.shape, a.patch, a.stride),
                     repeats=a.repeats, sync=torch.cuda.synchronize, out_json=a.json)
        print(f"[{res['name']}] volume {tuple(a.shape)}, patch {tuple(a.patch)}, stride {a.stride}, "
              f"{res['n_patches']} patches")
        print(f"  best {res['seconds'] * 1e3:9.2f} ms   ({res['us_per_patch']:8.3f} us/patch)   "
              f"first call {res['first_call'] * 1e3:.0f} ms")
        print(json.dumps(res))
    elif a.cmd == "rank-agreement":
        print(rank_table(rank_agreement(a.cases, tuple(a.forms.split(",")))))
    elif a.cmd == "summary":
        lines = []
        for f in a.files:
            for ln in open(f):
                ln = ln.strip()
                if ln.startswith("{"):
                    try:
                        d = json.loads(ln)
                    except json.JSONDecodeError:
                        continue
                    if "value" in d and "metric" in d:
                        lines.append(d)
        print(summary(lines))
    return 0


if __name__ == "__main__":
    sys.exit(main())
