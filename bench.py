"""Benchmark: R-MAT scale-22 triangle COUNT on B200 (learned vs heuristic
layouts), with the reference CPU engine as the baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one triangle COUNT query over the resident trie):
R-MAT scale 22, edge factor 16 (67,108,864 samples), a/b/c/d =
0.57/0.19/0.19/0.05, seed 42; symmetrised, self-loops dropped, deduped,
relabelled by degree, src < dst (64,152,167 rows).  The trie is built on
the device before timing (the reference's QUERY TIME excludes the load,
README.md:137).  The timed step is the generic-join bag: plan + intersection
kernel + count to host.  Every step's count is checked against the
reference engine's 2,110,948,863.

One JSON line on rank 0.  N > 1: every rank holds the trie, runs a
round-robin share of the work items, and the partial counts meet in one
8-byte NCCL all-reduce; time is the max over ranks.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EF, SEED = 22, 16, 42
ABCD = (0.57, 0.19, 0.19)
WORKLOAD = "R-MAT scale 22, edge factor 16, a/b/c/d 0.57/0.19/0.19/0.05, seed 42, degree-ordered src<dst; " \
           "triangle COUNT (TriangleAgg)"
METRIC = "R-MAT-22 triangle-count ms: learned vs heuristic layout on B200; CPU ref"


def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)["synthetic"]["rmat_s22_ef16_s42"]


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# --------------------------------------------------------------- CPU side
def run_reference(rows_src, rows_dst, repeats, threads=None, timeout=1800):
    from oracle import oracle as O
    if not O.ref_available():
        return None
    return O.ref_query_edges("triangle", rows_src, rows_dst, repeats=repeats, threads=threads, timeout=timeout)


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_arm(args):
    """The reference's own CPU engine (compiled from its sources) on the same
    workload, on all host cores.  Inputs come from the CPU oracle's generator
    (identical edge list, checked by sha1 in the tests)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    g = golden()
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/eh_ref was not built (no reference tree)"}))
        return 0
    u, v = O.gen_rmat(SEED, SCALE, EF << SCALE, *ABCD)
    s, d, _ = O.preprocess(u, v)
    del u, v
    r = run_reference(s, d, args.warmup + args.steps)
    times = r["query_s"][args.warmup:]
    assert r["count_u64"] == g["triangle"], r
    ms = [1e3 * x for x in times]
    value = statistics.median(ms)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "ms", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sum(ms) / len(ms), "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "uint32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "engine": "reference storage engine compiled from its sources "
                                                      "(oracle/_ref/eh_ref), generated-shape TriangleAgg bag",
                       "threads": r["threads"], "timer": "reference timer::stop_clock over the bag"},
            "count": r["count_u64"],
            "cpu_baseline": {"value": value, "unit": "ms", "cores": r["threads"], "kind": "reference",
                             "sample": "full workload, %d timed runs after %d warm-up" % (args.steps, args.warmup)},
            "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------- GPU side
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_record(layout):
    """Per-launch ncu figures of the intersection kernel at this workload for
    one layout policy (profiles/triangle_kernel_rmat22_<layout>_dram.json,
    written from a one-pass capture; see the .md beside it), or None."""
    p = os.path.join(ROOT, "profiles", "triangle_kernel_rmat22_%s_dram.json" % layout)
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def roofline(kernel_ms, alg_bytes, wedges, layout, peak, peak_kind, sm_mhz):
    """HBM roofline of the timed intersection kernel.  frac is measured DRAM
    traffic (ncu, same kernel, same layouts, per launch) over the kernel's
    CUDA-event time, against the measured copy peak.  The algorithmic bytes
    (both uint32 inputs of every pairwise intersection the reference loop
    nest evaluates) are reported beside it: most of them are served from
    shared memory and L2, so their rate is not a DRAM figure.  The issue
    side (warp instructions against 4 per SM per cycle) is what bounds this
    kernel."""
    rec = profile_record(layout)
    sec = kernel_ms * 1e-3
    out = {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
           "kernel": "eh::triangle_kernel<0> (MODE_COUNT)",
           "algorithmic_bytes": alg_bytes, "algorithmic_gbs": alg_bytes / sec / 1e9,
           "alg_over_peak": alg_bytes / sec / 1e9 / peak}
    if rec:
        traffic = int(rec["dram_bytes_read"]) + int(rec["dram_bytes_write"])
        out.update({"achieved": traffic / sec / 1e9, "frac": traffic / sec / 1e9 / peak, "traffic": traffic,
                    "traffic_source": "profiles/triangle_kernel_rmat22_%s_dram.json" % layout})
        inst = rec.get("warp_instructions")
        if inst:
            sms = int(rec.get("sms", 148))
            mhz = sm_mhz or float(rec.get("sm_mhz", 1965.0))
            issue_peak = 4.0 * sms * mhz * 1e6 * sec  # one warp instruction per SMSP per cycle
            out["issue"] = {"warp_instructions": int(inst), "per_candidate": int(inst) / max(1, wedges),
                            "issue_frac": int(inst) / issue_peak, "sm_mhz": mhz,
                            "note": "warp instructions per launch from the same capture; peak = 4 per SM per cycle"}
    else:
        out.update({"achieved": None, "frac": None, "traffic": None,
                    "traffic_source": "no capture of this kernel with %s layouts in profiles/" % layout})
    return out


# ------------------------------------------------------------------ timing
def timed_counts(tr, query, cfg, steps, warmup, want, flush, step_fn=None):
    """`warmup` untimed then `steps` timed runs of one query over a resident
    trie (engine CUDA events: plan + kernels + count to host), the L2 flushed
    between runs; every count is checked.  Returns (query ms list, kernel ms
    list, launches, last stats)."""
    import torch
    run = step_fn or (lambda: tr.count(query, stats=True, config=cfg))
    for _ in range(warmup):
        c, _ = run()
        assert c == want, (query, c, want)
    torch.cuda.synchronize()
    qms, kms, launches, st = [], [], 0, None
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        c, st = run()
        assert c == want, (query, c, want)
        qms.append(st["query_ms"])
        kms.append(st["kernel_ms"])
        launches += st["launches"]
    return qms, kms, launches, st


def _ms(x):
    return {"mean_ms": statistics.mean(x), "median_ms": statistics.median(x)}


# --------------------------------------------------- the other workloads
def other_workloads(E, ctx, args, flush, deadline, model22):
    """The other benchmark workloads beside the headline: the 256-graph batch, the
    R-MAT-20 4-clique, Chung-Lu 2^23 lollipop and barbell; each with the
    density-rule and learned layouts on the device (identical counts) and the
    reference engine on this host's cores (in the same run) on a stated
    sample.  Skipped once `deadline` (time.time()) has passed."""
    import numpy as np
    from emptyheaded_b200 import autotune as AT, learn, workloads as W
    from oracle import oracle as O
    gold = W.golden_counts()
    out = {}
    ref_ok = O.ref_available()
    steps = max(3, min(args.steps, 5))

    def over():
        return time.time() > deadline

    # ---- 256 R-MAT graphs (scales 10..18), triangle COUNT, one CUDA-graph replay
    if not over():
        try:
            spec = W.batch256_spec()
            want = [int(x["triangle"]) for x in json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))
                    ["batch256"]]
            tries = [W.build_rmat_trie(E, sc, sd, ctx=ctx) for sc, sd in spec]

            def run_batch(tag):
                b = E.Batch(tries)
                res = b.run()
                assert [int(x) for x in res] == want, tag
                ms = []
                for _ in range(steps):
                    flush.zero_()
                    torch_sync()
                    r, st = b.run(stats=True)
                    assert [int(x) for x in r] == want, tag
                    ms.append(st["query_ms"])
                b.free()
                return ms

            t_leg = time.time()
            ms_h = run_batch("heuristic")
            # a model trained on the batch's own logs: the even-numbered graphs
            # are profiled, the odd-numbered ones are never seen in training
            mb, infob, _ = learn.train_from_tries(E, tries[::2], passes=1, epochs=30, config=dict(AT.DEFAULT))
            for t in tries:
                t.relayout(policy=E.LEARNED, model=mb)
            ms_l = run_batch("learned")
            # the density rule as judge, graph by graph: each keeps the faster layouts
            kept = [learn.judge(E, t, mb, config=dict(AT.DEFAULT), reps=2)["kept"] for t in tries]
            ms_j = run_batch("judged")
            mb.free()
            rows = int(sum(t.info()["rows"] for t in tries))
            for t in tries:
                t.free()
            rec = {"graphs": len(spec), "rows": rows, "launches_per_run": 1, "heuristic": _ms(ms_h),
                   "learned": _ms(ms_l), "learned_speedup": statistics.mean(ms_h) / statistics.mean(ms_l),
                   "judged": _ms(ms_j), "judged_speedup": statistics.mean(ms_h) / statistics.mean(ms_j),
                   "judged_learned_graphs": kept.count("learned"),
                   "model": dict({k: infob[k] for k in ("median_abs_pct_error", "regret_learned_pct",
                                                        "regret_heuristic_pct", "train_rows") if k in infob},
                                 trained_on="the batch's even-numbered graphs (128); odd-numbered held out")}
            if ref_ok and not args.no_cpu:
                # the reference engine graph by graph until ~20 s of its query time; scaled to all rows
                t0, q, done_rows, done = time.time(), 0.0, 0, 0
                order = list(range(len(spec)))
                for i in order:
                    sc, sd = spec[i]
                    u, v = O.gen_rmat(sd, sc, 16 << sc, *ABCD)
                    s_, d_, _ = O.preprocess(u, v)
                    r = O.ref_query_edges("triangle", s_, d_, repeats=1, timeout=300)
                    assert r["count_u64"] == want[i]
                    q += r["query_s"][0]
                    done_rows += len(s_)
                    done += 1
                    if time.time() - t0 > 25 or over():
                        break
                rec["cpu_baseline"] = {"value": 1e3 * q * rows / max(1, done_rows), "unit": "ms",
                                       "cores": r["threads"], "kind": "reference",
                                       "sample": "%d of %d graphs (%d of %d rows), query time summed and scaled "
                                                 "by rows" % (done, len(spec), done_rows, rows)}
            rec["wall_s"] = round(time.time() - t_leg, 1)
            out["batch256_triangle"] = rec
        except Exception as ex:
            out["batch256_triangle"] = {"error": repr(ex)[:300]}

    # ---- R-MAT-20 4-clique: a cost model trained on the 4-clique kernel's own logs
    if not over():
        try:
            want = int(gold["rmat_s20_ef16_s42"]["clique4"])
            t_leg = time.time()
            t = W.build_rmat_trie(E, 20, SEED, ctx=ctx)
            cfg = dict(AT.DEFAULT)
            qh, kh, _, _ = timed_counts(t, "clique4", cfg, steps, 2, want, flush)
            m4, info4, prof4 = learn.train_from_trie(E, t, passes=1, epochs=40, query="clique4", config=cfg)
            t.relayout(policy=E.LEARNED, model=m4)
            ql, kl, _, _ = timed_counts(t, "clique4", cfg, steps, 2, want, flush)
            t.relayout(policy=E.EXPLICIT, layouts=learn.best_layouts(prof4))
            qb, _, _, _ = timed_counts(t, "clique4", cfg, steps, 2, want, flush)
            j4 = learn.judge(E, t, m4, query="clique4", config=cfg)
            qj, _, _, _ = timed_counts(t, "clique4", cfg, steps, 2, want, flush)
            rec = {"rows": t.info()["rows"], "count": want, "heuristic": _ms(qh), "learned": _ms(ql),
                   "exhaustive_best": _ms(qb), "learned_speedup": statistics.mean(qh) / statistics.mean(ql),
                   "judged": dict(_ms(qj), kept=j4["kept"]),
                   "model": {k: info4[k] for k in ("median_abs_pct_error", "regret_learned_pct",
                                                  "regret_heuristic_pct", "sets_staged") if k in info4}}
            t.free()
            m4.free()
            if ref_ok and not args.no_cpu and not over():
                u, v = O.gen_rmat(SEED, 20, 16 << 20, *ABCD)
                s_, d_, _ = O.preprocess(u, v)
                r = O.ref_query_edges("clique4", s_, d_, repeats=1, timeout=600)
                assert r["count_u64"] == want
                rec["cpu_baseline"] = {"value": 1e3 * r["query_s"][0], "unit": "ms", "cores": r["threads"],
                                       "kind": "reference", "sample": "full R-MAT-20 4-clique COUNT, one run, "
                                                                      "trie build excluded"}
            rec["wall_s"] = round(time.time() - t_leg, 1)
            out["rmat20_clique4"] = rec
        except Exception as ex:
            out["rmat20_clique4"] = {"error": repr(ex)[:300]}

    # ---- Chung-Lu 2^23 lollipop / barbell: a model trained on the annotated pass's logs
    if not over():
        try:
            t_leg = time.time()
            g23 = gold["chunglu_n8388608_d32_g2.1_s9_sym"]
            t = W.build_chunglu_trie(E, ctx=ctx)
            cfg = dict(AT.DEFAULT)
            rec = {"rows": t.info()["rows"]}
            res = {}
            for q in ("lollipop", "barbell"):
                res[q] = timed_counts(t, q, cfg, 3, 1, int(g23[q]), flush)[0]
            mc, infoc, _ = learn.train_from_trie(E, t, passes=1, epochs=40, query="lollipop", config=cfg)
            t.relayout(policy=E.LEARNED, model=mc)
            for q in ("lollipop", "barbell"):
                ql = timed_counts(t, q, cfg, 3, 1, int(g23[q]), flush)[0]
                rec[q] = {"count": int(g23[q]), "heuristic": _ms(res[q]), "learned": _ms(ql),
                          "learned_speedup": statistics.mean(res[q]) / statistics.mean(ql)}
            jc = learn.judge(E, t, mc, query="lollipop", config=cfg, reps=2)
            rec["judged_kept"] = jc["kept"]
            rec["model"] = {k: infoc[k] for k in ("median_abs_pct_error", "regret_learned_pct",
                                                  "regret_heuristic_pct", "sets_staged") if k in infoc}
            t.free()
            mc.free()
            if ref_ok and not args.no_cpu and not over():
                # the reference engine on a bounded sample: the same generator at n = 2^19
                # (its queries at 2^23 take minutes); the device on the same sample beside it
                n = 1 << 19
                u, v = O.gen_chunglu(9, n, n * 16, 2.1)
                s_, d_, _ = O.preprocess(u, v, symmetric=True)
                ts = E.Trie(s_, d_, ctx=ctx)
                for q in ("lollipop", "barbell"):
                    r = O.ref_query_edges(q, s_, d_, repeats=1, timeout=600)
                    dev = timed_counts(ts, q, cfg, 3, 1, r["count_u64"], flush)[0]
                    rec[q]["cpu_baseline"] = {"value": 1e3 * r["query_s"][0], "unit": "ms", "cores": r["threads"],
                                              "kind": "reference",
                                              "sample": "Chung-Lu n=2^19 (same generator, average degree 32, "
                                                        "exponent 2.1), one run; device on the same sample: "
                                                        "%.2f ms (density rule)" % statistics.mean(dev)}
                ts.free()
            rec["wall_s"] = round(time.time() - t_leg, 1)
            out["chunglu23_lollipop_barbell"] = rec
        except Exception as ex:
            out["chunglu23_lollipop_barbell"] = {"error": repr(ex)[:300]}
    return out


def torch_sync():
    import torch
    torch.cuda.synchronize()


def ours_arm(args):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    import emptyheaded_b200 as E
    from emptyheaded_b200 import autotune as AT, learn, shard as SH, workloads as W

    t_start = time.time()
    ctx = E.Context(local if world > 1 else 0)
    E._default = ctx
    g = golden()
    want = g["triangle"]
    # ---- input pipeline and trie build (untimed, like the reference's load)
    t0 = time.time()
    u, v = E.gen_rmat(SEED, SCALE, EF << SCALE, *ABCD, ctx=ctx)
    s, d, nodes = E.preprocess(u, v, ctx=ctx)
    u.free()
    v.free()
    trie = E.Trie(s, d, ctx=ctx)
    info_h = trie.info()
    build_s = time.time() - t0
    shard = (rank, world)
    flush = torch.empty(64 << 20, dtype=torch.int32, device="cuda")  # 256 MB > L2

    def step(cfg):
        c, st = trie.count("triangle", stats=True, shard=shard, config=cfg)
        if world > 1:
            c = SH.combine_counts(c, device="cuda")
        return c, st

    def tune():
        # every rank must cut the same plan (the chunk size sets the items)
        return dict(AT.DEFAULT) if world > 1 else AT.tune(trie)[0]

    def timed(cfg):
        if world > 1:
            torch.distributed.barrier()
        r = timed_counts(trie, "triangle", cfg, args.steps, args.warmup, want, flush, lambda: step(cfg))
        if world > 1:
            torch.distributed.barrier()
        return r

    def rmax(x):
        return x if world == 1 else SH.max_over_ranks(x, device="cuda")

    # ---- density-rule layouts (schedule autotuned for them, untimed)
    cfg_h = tune()
    # clocks are sampled over the device-timed steps only: nvidia-smi's driver
    # queries stall host-side CUDA calls, which the e2e leg measures
    args.sampler.start()
    qh, kh, lh, st_h = timed(cfg_h)
    # ---- learned layouts: the cost model trained on this engine's logged timings
    learn_info, extra_layouts = {}, {}
    model = None
    cfg_l, ql, kl, ll, st_l = cfg_h, qh, kh, lh, st_h
    try:
        if world > 1:
            # every rank must cut the same plan from the same layouts and
            # predicted costs: rank 0 trains the model, the others load its
            # parameters (the same collectives on every rank, failure included)
            ok = torch.zeros(1, device="cuda")
            model = E.Model(learn.DIMS, ctx=ctx)
            if rank == 0:
                try:
                    model, learn_info, _ = learn.train_from_trie(E, trie, passes=1)
                    ok.fill_(1)
                except Exception as ex:
                    learn_info = {"error": repr(ex)[:300]}
            torch.distributed.broadcast(ok, 0)
            if ok.item() != 1:
                raise RuntimeError("cost model training failed on rank 0")
            p = torch.from_numpy(model.params()).cuda()
            torch.distributed.broadcast(p, 0)
            model.set_params(p.cpu().numpy())
        else:
            prof = learn.profile(E, trie, reps=2, config=cfg_h)
            model, learn_info, _ = learn.train_from_trie(E, trie, prof=prof)
            learn_info["evaluated_on"] = "the R-MAT-22 profile it was trained on (in sample)"
            # a model trained on another graph (R-MAT-20), judged on this one
            t20 = W.build_rmat_trie(E, 20, SEED, ctx=ctx)
            model_ho, info20, _ = learn.train_from_trie(E, t20, passes=2, config=cfg_h)
            t20.free()
            ho = learn.evaluate(E, model_ho, prof)
            ho["trained_on"] = "R-MAT-20 seed 42 triangle logs; evaluated on the R-MAT-22 profile (held out)"
            trie.relayout(policy=E.LEARNED, model=model_ho)
            cfg_ho = tune()
            qo, ko, _, _ = timed(cfg_ho)
            ho.update({"query": _ms(qo), "kernel": _ms(ko), "speedup_vs_heuristic": statistics.mean(qh) /
                       statistics.mean(qo), "layout_hist": _hist(trie.info())})
            extra_layouts["learned_held_out"] = ho
            # the per-set exhaustive search's own assignment: the ceiling of any layout policy
            trie.relayout(policy=E.EXPLICIT, layouts=learn.best_layouts(prof))
            cfg_b = tune()
            qb, kb, _, _ = timed(cfg_b)
            extra_layouts["exhaustive_best"] = {"query": _ms(qb), "kernel": _ms(kb), "schedule": cfg_b,
                                                "speedup_vs_heuristic": statistics.mean(qh) / statistics.mean(qb),
                                                "layout_hist": _hist(trie.info())}
            model_ho.free()
        trie.relayout(policy=E.LEARNED, model=model)
        learn_info["layout_hist"] = _hist(trie.info())
        cfg_l = tune()
        ql, kl, ll, st_l = timed(cfg_l)
    except Exception as ex:  # the learned arm must not hide the measurement
        learn_info = {"error": repr(ex)[:300]}
        model = None
    clocks = args.sampler.stop()

    ms_h, ms_l = rmax(statistics.mean(qh)), rmax(statistics.mean(ql))
    kern_h, kern_l = rmax(statistics.mean(kh)), rmax(statistics.mean(kl))
    med_h, med_l = rmax(statistics.median(qh)), rmax(statistics.median(ql))

    # ---- e2e through the host-buffer entry: CSR in pinned host memory,
    # copied to the device every step (plus the trie index build), count back
    e2e = None
    if world == 1:
        head, off, vals, _ = trie.export()
        head_p = torch.from_numpy(head).pin_memory().numpy()
        off_p = torch.from_numpy(off.view(np.int64)).pin_memory().numpy().view(np.uint64)
        vals_p = torch.from_numpy(vals.view(np.int32)).pin_memory().numpy().view(np.uint32)
        h2d = head_p.nbytes + off_p.nbytes + vals_p.nbytes
        pol = E.LEARNED if model is not None else E.HEURISTIC
        # one call measures its peak device memory; the pool then keeps that
        # much (plus slack) as one block, so no timed call maps new memory
        used0 = ctx.memory()["used"]
        ctx.reserve(0)
        c = E.count_host_csr(head_p, off_p, vals_p, nodes, policy=pol, model=model, ctx=ctx, config=cfg_l)
        assert c == want
        pool_bytes = int(1.1 * (ctx.memory()["peak"] - used0)) + (64 << 20)
        ctx.reserve(pool_bytes)
        for _ in range(max(3, args.warmup)):
            c = E.count_host_csr(head_p, off_p, vals_p, nodes, policy=pol, model=model, ctx=ctx, config=cfg_l)
            assert c == want
        ev = []
        for _ in range(max(3, args.steps)):
            torch.cuda.synchronize()
            a = time.perf_counter()
            c = E.count_host_csr(head_p, off_p, vals_p, nodes, policy=pol, model=model, ctx=ctx, config=cfg_l)
            ev.append(1e3 * (time.perf_counter() - a))
            assert c == want
        e2e = {"value": statistics.median(ev), "unit": "ms", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 8,
               "path": "eh_query_count_host_csr: pinned host CSR -> device, trie index + layouts, count, result to host",
               "runs_ms": [round(x, 2) for x in ev], "pool_reserved_bytes": pool_bytes}

    # ---- CPU baseline (rank 0, N = 1): the reference engine on the same rows
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        hs, hd = s.numpy(), d.numpy()
        try:
            r = run_reference(hs, hd, 3)
            if r:
                cpu = {"value": 1e3 * statistics.median(r["query_s"]), "unit": "ms", "cores": r["threads"],
                       "kind": "reference",
                       "sample": "full R-MAT-22 triangle COUNT, median of 3 runs, trie build excluded "
                                 "(reference build %.1f s, sort serialised)" % r["build_s"],
                       "count": r["count_u64"]}
                assert r["count_u64"] == want
        except Exception as ex:
            cpu = {"value": None, "unit": "ms", "cores": cpu_threads(), "kind": "reference", "sample": repr(ex)[:200]}
    s.free()
    d.free()
    trie.free()

    # ---- the other benchmark workloads beside the headline (single GPU)
    workloads = None
    if world == 1 and not args.no_extra and model is not None:
        workloads = other_workloads(E, ctx, args, flush, t_start + args.budget_s, model)

    if rank == 0:
        peak, peak_kind = load_peaks()
        layout_name = "learned" if model is not None else "heuristic"
        roof = roofline(kern_l, st_l["algorithmic_bytes"], st_l["wedges"], layout_name, peak,
                        peak_kind + " (hbm_gbs)", clocks.get("sm_mhz"))
        line = {
            "metric": METRIC, "value": ms_l, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_l, "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "uint32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows": info_h["rows"], "nodes": nodes, "layout": layout_name,
                       "heuristic_ms": ms_h, "learned_ms": ms_l, "learned_speedup": ms_h / ms_l,
                       "heuristic_kernel_ms": kern_h, "learned_kernel_ms": kern_l,
                       "heuristic_median_ms": med_h, "learned_median_ms": med_l,
                       "l2": "trie (%.2f GB) larger than L2, and a 256 MB buffer written between steps"
                             % (info_h["device_bytes"] / 1e9),
                       "trie_build_s": build_s, "parallelism": "shards of work items" if world > 1 else "single GPU",
                       "schedule_heuristic": cfg_h, "schedule_learned": cfg_l,
                       "learned": learn_info, "layouts_compared": extra_layouts},
            "count": want,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(ll / max(1, args.steps)) * args.steps,
            "workloads": workloads,
        }
        line["clocks"] = clocks
        line["wall_s"] = round(time.time() - t_start, 1)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def _hist(info):
    return {"uint": info["n_uinteger"], "bitset": info["n_range_bitset"], "block": info["n_block_bitset"],
            "bitset_words": info["bitset_words"], "device_bytes": info["device_bytes"]}


def case_arm(args):
    """A small self-checking query case for profiler captures (not a bench
    line): builds the R-MAT trie of --scale on the device, lays it out with
    --layout (learned: the cost model is trained on this trie first), and
    runs the query --repeat times inside the NVTX range "case", printing the
    counts and device times.  Captures select the case's launches with
    --nvtx --nvtx-include "case/"."""
    import torch
    import emptyheaded_b200 as E
    from emptyheaded_b200 import learn, workloads as W

    t = W.build_rmat_trie(E, args.scale, SEED)
    forced = {"uint": E.UINTEGER, "bitset": E.RANGE_BITSET, "block": E.BLOCK_BITSET}
    learn_info = None
    cfg = {k: v for k, v in (("smem_words", args.smem_words), ("warps", args.warps), ("chunk", args.chunk),
                             ("long_row", args.long_row)) if v}
    cfg["block_items"] = not args.no_block_items
    if args.layout == "learned":
        model, learn_info, _ = learn.train_from_trie(E, t, config=cfg)
        t.relayout(policy=E.LEARNED, model=model)
    elif args.layout in forced:
        t.relayout(policy=E.FORCED, forced=forced[args.layout], max_bitset_bytes=1 << 50)
    runs = []
    t.count(args.query, config=cfg)  # warm
    torch.cuda.nvtx.range_push("case")
    for _ in range(args.repeat):
        c, st = t.count(args.query, stats=True, config=cfg)
        runs.append({"count": c, "query_ms": st["query_ms"], "kernel_ms": st["kernel_ms"], "wedges": st["wedges"],
                     "algorithmic_bytes": st["algorithmic_bytes"]})
    torch.cuda.nvtx.range_pop()
    g = W.golden_counts().get("rmat_s%d_ef16_s%d" % (args.scale, SEED), {})
    ok = all(r["count"] == g[args.query] for r in runs) if args.query in g else None
    print(json.dumps({"case": "rmat%d" % args.scale, "query": args.query, "layout": args.layout, "ok": ok,
                      "schedule": cfg,
                      "info": t.info(), "learned": learn_info, "runs": runs}))
    t.free()
    return 0 if ok in (None, True) else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline legs")
    ap.add_argument("--no-extra", action="store_true", help="headline only: skip the batch, 4-clique and lollipop/barbell workloads")
    ap.add_argument("--budget-s", type=float, default=420.0,
                    help="wall-clock budget after which the remaining other configs are skipped")
    ap.add_argument("--case", action="store_true", help="profiler case instead of the bench line")
    ap.add_argument("--scale", type=int, default=20, help="--case: R-MAT scale")
    ap.add_argument("--layout", default="heuristic", choices=["heuristic", "learned", "uint", "bitset", "block"],
                    help="--case: layout policy")
    ap.add_argument("--query", default="triangle", help="--case: query")
    ap.add_argument("--repeat", type=int, default=2, help="--case: runs inside the NVTX range")
    ap.add_argument("--no-block-items", action="store_true", help="--case: stage every N(b) per warp")
    ap.add_argument("--smem-words", type=int, default=0, help="--case: staging words per warp")
    ap.add_argument("--warps", type=int, default=0, help="--case: warps per block")
    ap.add_argument("--chunk", type=int, default=0, help="--case: probes per work item")
    ap.add_argument("--long-row", type=int, default=0, help="--case: rows at least this long run warp-wide")
    args = ap.parse_args()
    if args.case:
        return case_arm(args)
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return reference_arm(args)
    _, _, local = dist_env()
    args.sampler = ClockSampler(local)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
