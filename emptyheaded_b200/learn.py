"""Learned layout policy: profile, train, evaluate.

The engine logs, for every work item of a triangle query, the SM cycles it
spent on the staged set N(b) under the layout that set had
(eh_timing_records).  `profile` runs the query once per candidate layout
(uint / range bitset / block bitset, each set forced where admissible) and
sums the cycles per set: for every set this is an exhaustive layout search.
`train` fits the cost model (the engine's fp32 MLP, trained on the GPU by
its own kernels) to predict log cycles from the set's features and a
layout; EH_POLICY_LEARNED then gives each set its predicted-cheapest
layout.  The reference's density rule (common::is_sparse,
utils/common.hpp:60-66) stays as the fallback for sets the plan never
stages and as the point of comparison: `evaluate` reports the model's prediction error
and the regret of both policies against the exhaustive search.
"""
import numpy as np

UINT, BITSET, BLOCK = 1, 0, 3
LAYOUTS = (UINT, BITSET, BLOCK)
DIMS = [6, 32, 32, 1]
# per-set cap used when forcing range bitsets for profiling: the same
# admission the learned chooser applies (16 words per element + 64)
REL_WORDS, ABS_WORDS = 16, 64


def set_features(head_len, rng, pairs, layout):
    """Features of a set for the model (fp32): log1p(len), log1p(range),
    density len/(range+1), log1p(pairs probed against it), layout one-hot
    (bitset, block); uint is the zero vector.  Matches model_features in
    csrc/eh_model.cu."""
    f = np.zeros((len(head_len), 6), np.float32)
    f[:, 0] = np.log1p(head_len)
    f[:, 1] = np.log1p(rng)
    f[:, 2] = head_len / (rng + 1.0)
    f[:, 3] = np.log1p(pairs)
    f[:, 4] = layout == BITSET
    f[:, 5] = layout == BLOCK
    return f


def profile(E, trie, reps=2, query="triangle", config=None):
    """Per-set cycles of `query`'s intersection kernel under each layout
    (the triangle or 4-clique kernel; for lollipop / barbell, the annotated
    triangle pass that dominates them).  Returns (len, range, pairs,
    cycles[layout] with NaN where the layout was not admissible, base
    heuristic layout).  `config` is the schedule (autotune dict) the timed
    runs will use: costs depend on it (the staging capacity per warp above
    all), so the profile runs with the same one."""
    head, off, vals, heur = trie.export()
    n = len(head)
    lens = np.diff(off).astype(np.float64)
    first = vals[off[:-1].astype(np.int64)].astype(np.float64)
    last = vals[np.maximum(off[1:].astype(np.int64) - 1, 0)].astype(np.float64)
    rng = np.where(lens > 0, last - first, 0.0)
    words = np.floor(last / 64) - np.floor(first / 64) + 1
    cycles = {}
    pairs = np.zeros(n)
    for L in LAYOUTS:
        if L == BITSET:
            # admission per set as in the learned chooser (16 words per
            # element + 64); the absolute cap is set out of the way
            trie.relayout(policy=E.FORCED, forced=BITSET, max_bitset_bytes=1 << 50)
            ok = words <= REL_WORDS * lens + ABS_WORDS
        else:
            trie.relayout(policy=E.FORCED, forced=L)
            ok = np.ones(n, bool)
        _, _, _, lay = trie.export()
        acc = np.zeros(n)
        for _ in range(reps):
            trie.count(query, record=True, config=config)
            rec = E.timing_records(trie.ctx)
            hb = rec[:, 6].view(np.uint32).astype(np.int64)
            acc += np.bincount(hb, weights=rec[:, 7].astype(np.float64), minlength=n)
            pairs = np.bincount(hb, weights=rec[:, 1].astype(np.float64), minlength=n)
        c = acc / reps
        c[(lay != L) | ~ok] = np.nan
        cycles[L] = c
    trie.relayout()
    return dict(lens=lens, range=rng, pairs=pairs, cycles=cycles, heuristic=heur.astype(np.int64), words=words)


def dataset(prof, max_weight=32, max_rows=2_000_000, seed=0):
    """Training rows (features, log1p cycles), one per staged set and
    admissible layout.  A set's row is repeated in proportion to its cost
    (at most max_weight times): the sets that hold the time are the ones the
    choice has to get right, and most sets are cheap.  Above max_rows rows
    a seeded uniform sample of max_rows is kept (training time grows with
    the rows; a power-law graph has millions of staged sets)."""
    xs, ys = [], []
    staged = prof["pairs"] > 0
    for L in LAYOUTS:
        c = prof["cycles"][L]
        m = staged & np.isfinite(c) & (c > 0)
        if not m.any():
            continue
        reps = np.clip(np.round(c[m] / c[m].mean()), 1, max_weight).astype(np.int64)
        f = set_features(prof["lens"][m], prof["range"][m], prof["pairs"][m], np.full(m.sum(), L))
        y = np.log1p(c[m]).astype(np.float32)[:, None]
        xs.append(np.repeat(f, reps, axis=0))
        ys.append(np.repeat(y, reps, axis=0))
    x, y = np.concatenate(xs), np.concatenate(ys)
    if max_rows and len(x) > max_rows:
        keep = np.sort(np.random.default_rng(seed).choice(len(x), max_rows, replace=False))
        x, y = x[keep], y[keep]
    return x, y


def on_policy_rows(E, trie, model, query="triangle", config=None, explore=0.5, seed=0, reps=1):
    """Per-set cycles under a mixed assignment.  The forced-layout profile
    times every set while all others share its layout; the model's own
    assignment mixes layouts, and a set's cost depends on its neighbours'
    (word-level rows need both sides in range bitsets, the annotated pass
    counts matches in shared memory only for some staged forms).  The trie
    is laid out by the model, a random `explore` share of the sets it moved
    goes back to the density rule's layout, the query runs with records, and
    each staged set's cycles come back with the layout it really had.
    Returns (features, log1p cycles); the trie is left with the rule's
    layouts."""
    trie.relayout()
    head, off, vals, heur = trie.export()
    trie.relayout(policy=E.LEARNED, model=model)
    _, _, _, lay = trie.export()
    rng = np.random.default_rng(seed)
    moved = lay != heur
    back = moved & (rng.random(len(lay)) < explore)
    lay = np.where(back, heur, lay).astype(np.uint8)
    trie.relayout(policy=E.EXPLICIT, layouts=lay)
    n = len(head)
    acc = np.zeros(n)
    pairs = np.zeros(n)
    for _ in range(reps):
        trie.count(query, record=True, config=config)
        rec = E.timing_records(trie.ctx)
        hb = rec[:, 6].view(np.uint32).astype(np.int64)
        acc += np.bincount(hb, weights=rec[:, 7].astype(np.float64), minlength=n)
        pairs = np.bincount(hb, weights=rec[:, 1].astype(np.float64), minlength=n)
    trie.relayout()
    lens = np.diff(off).astype(np.float64)
    first = vals[off[:-1].astype(np.int64)].astype(np.float64)
    last = vals[np.maximum(off[1:].astype(np.int64) - 1, 0)].astype(np.float64)
    rg = np.where(lens > 0, last - first, 0.0)
    m = (pairs > 0) & (acc > 0)
    f = set_features(lens[m], rg[m], pairs[m], lay[m].astype(np.int64))
    return f, np.log1p(acc[m] / reps).astype(np.float32)[:, None]


def refine(E, trie, model, prof, query="triangle", config=None, rounds=1, epochs=40, weight=4, seed=0):
    """Retrain on the forced-layout profile plus on-policy rows
    (on_policy_rows, repeated `weight` times) gathered under the current
    model's assignment, `rounds` times.  Returns (model, info) with info
    evaluated on the forced profile as before."""
    x0, y0 = dataset(prof)
    xs, ys = [x0], [y0]
    for r in range(rounds):
        f, y = on_policy_rows(E, trie, model, query=query, config=config, seed=seed + r)
        xs.append(np.repeat(f, weight, axis=0))
        ys.append(np.repeat(y, weight, axis=0))
        model.free()
        model, _ = train(E, np.concatenate(xs), np.concatenate(ys), ctx=trie.ctx, epochs=epochs, seed=seed + r)
    info = evaluate(E, model, prof)
    info["on_policy_rows"] = int(sum(len(x) for x in xs[1:]) // max(1, weight))
    info["query"] = query
    return model, info


def _fold(params, dims, mu_x, sd_x, mu_y, sd_y):
    """Fold input standardisation into layer 0 and output scaling into the
    last layer, so the device chooser evaluates the model on raw features."""
    p = params.astype(np.float64).copy()
    d0, d1 = dims[0], dims[1]
    W0 = p[: d1 * d0].reshape(d1, d0)
    b0 = p[d1 * d0: d1 * d0 + d1]
    b0 -= W0 @ (mu_x / sd_x)
    W0 /= sd_x[None, :]
    o = 0
    for l in range(len(dims) - 1):
        o += dims[l + 1] * dims[l] + dims[l + 1]
    dl, dp = dims[-1], dims[-2]
    WL = p[o - dl - dl * dp: o - dl].reshape(dl, dp)
    bL = p[o - dl: o]
    WL *= sd_y
    bL *= sd_y
    bL += mu_y
    return p.astype(np.float32)


def train(E, x, y, ctx=None, epochs=40, batch=2048, lr=0.05, seed=0):
    """SGD on the device (eh_model_train) over shuffled minibatches of
    standardised features and targets; returns the model with the
    standardisation folded into its weights."""
    model = E.Model(DIMS, seed=seed, ctx=ctx)
    mu_x = x.mean(0).astype(np.float64)
    sd_x = x.std(0).astype(np.float64)
    sd_x[sd_x < 1e-6] = 1.0
    mu_y, sd_y = float(y.mean()), float(y.std()) or 1.0
    xn = ((x - mu_x) / sd_x).astype(np.float32)
    yn = ((y - mu_y) / sd_y).astype(np.float32)
    rng = np.random.default_rng(seed)
    n = len(x)
    losses = []
    for ep in range(epochs):
        perm = rng.permutation(n)
        step_lr = lr * (0.1 if ep >= int(0.75 * epochs) else 1.0)
        for i in range(0, n, batch):
            idx = perm[i:i + batch]
            if len(idx) < 16:
                continue
            losses.append(model.train(xn[idx], yn[idx], lr=step_lr, steps=1))
    model.set_params(_fold(model.params(), DIMS, mu_x, sd_x, mu_y, sd_y))
    return model, losses


MIN_GAIN = 0.1  # the device chooser's default margin (eh_layout_config.min_gain = 0)


def evaluate(E, model, prof, min_gain=MIN_GAIN):
    """Prediction error and regret against the per-set exhaustive search.
    The model's choice is the device chooser's: its predicted-cheapest
    admissible layout, unless that is predicted to gain less than min_gain
    over the density rule's layout, which then stays."""
    staged = prof["pairs"] > 0
    n = len(prof["lens"])
    C = np.stack([prof["cycles"][L] for L in LAYOUTS], 1)  # n x 3
    best = np.nanmin(np.where(np.isfinite(C), C, np.inf), 1)
    # model choice among admissible layouts
    preds = []
    for L in LAYOUTS:
        f = set_features(prof["lens"], prof["range"], prof["pairs"], np.full(n, L))
        preds.append(model.predict(f)[:, 0])
    P = np.stack(preds, 1)
    P = np.where(np.isfinite(C), P, np.inf)
    choice = np.argmin(P, 1)
    heur_col = np.where(prof["heuristic"] == BITSET, 1, 0)  # heuristic uses uint or bitset
    rows = np.arange(n)
    keep = (choice != heur_col) & ~(P[rows, choice] < P[rows, heur_col] + np.log1p(-min_gain))
    choice = np.where(keep & np.isfinite(P[rows, heur_col]), heur_col, choice)
    chosen = C[rows, choice]
    heur_cost = C[rows, heur_col]
    m = staged & np.isfinite(best) & np.isfinite(chosen) & np.isfinite(heur_cost)
    total_best = best[m].sum()
    finite = np.isfinite(C) & (C > 0)
    err = np.abs(np.expm1(P[finite]) - C[finite]) / C[finite]
    return {
        "sets_staged": int(staged.sum()),
        "median_abs_pct_error": float(np.median(err) * 100) if err.size else None,
        "regret_learned_pct": float((chosen[m].sum() / total_best - 1) * 100) if total_best else None,
        "regret_heuristic_pct": float((heur_cost[m].sum() / total_best - 1) * 100) if total_best else None,
        "choice_hist": {"uint": int((choice[staged] == 0).sum()), "bitset": int((choice[staged] == 1).sum()),
                        "block": int((choice[staged] == 2).sum())},
    }


def judge(E, trie, model, query="triangle", config=None, reps=3):
    """The density rule as judge: `query` timed on `trie` (engine CUDA
    events, kernel time, median of `reps` after one warm run) with the
    rule's layouts and with the model's; the trie keeps the faster
    assignment.  Layouts change speed only: every count is checked against
    the first.  Returns {heuristic_ms, learned_ms, kept}."""
    import statistics
    want = [None]

    def timed():
        ks = []
        for _ in range(reps + 1):
            c, st = trie.count(query, stats=True, config=config)
            if want[0] is None:
                want[0] = c
            if c != want[0]:
                raise AssertionError("layouts changed the count: %d != %d" % (c, want[0]))
            ks.append(st["kernel_ms"])
        return statistics.median(ks[1:])

    trie.relayout()
    h = timed()
    trie.relayout(policy=E.LEARNED, model=model)
    l = timed()
    kept = "learned" if l <= h else "heuristic"
    if kept == "heuristic":
        trie.relayout()
    return {"heuristic_ms": h, "learned_ms": l, "kept": kept}


def best_layouts(prof):
    """The per-set exhaustive search's assignment: each staged set's
    cheapest admissible layout by the profiled cycles, the density rule for
    the sets no plan stages (EH_POLICY_EXPLICIT takes it)."""
    C = np.stack([prof["cycles"][L] for L in LAYOUTS], 1)
    C = np.where(np.isfinite(C) & (C > 0), C, np.inf)
    pick = np.asarray(LAYOUTS, np.uint8)[np.argmin(C, 1)]
    staged = (prof["pairs"] > 0) & np.isfinite(C.min(1))
    return np.where(staged, pick, prof["heuristic"].astype(np.uint8)).astype(np.uint8)


def merge_profiles(profs):
    """One profile over the sets of several tries (a batch's graphs)."""
    out = {k: np.concatenate([p[k] for p in profs]) for k in ("lens", "range", "pairs", "heuristic", "words")}
    out["cycles"] = {L: np.concatenate([p["cycles"][L] for p in profs]) for L in LAYOUTS}
    return out


def train_from_tries(E, tries, passes=2, epochs=60, query="triangle", config=None):
    """train_from_trie over many tries: each is profiled on its own (the
    engine's per-item logs of its own runs), the logs are pooled and one
    model is trained on them.  Returns (model, info, pooled profile)."""
    prof = merge_profiles([profile(E, t, reps=passes, query=query, config=config) for t in tries])
    x, y = dataset(prof)
    model, losses = train(E, x, y, ctx=tries[0].ctx, epochs=epochs)
    info = evaluate(E, model, prof)
    info["train_rows"] = int(len(x))
    info["final_loss"] = float(np.mean(losses[-20:])) if losses else None
    info["query"] = query
    info["tries"] = len(tries)
    return model, info, prof


def train_from_trie(E, trie, passes=2, epochs=60, query="triangle", prof=None, config=None):
    """Profile `trie` (or take its profile), train the cost model on the
    logs, evaluate it on the same logs.  Returns (model, info, profile)."""
    prof = prof if prof is not None else profile(E, trie, reps=passes, query=query, config=config)
    x, y = dataset(prof)
    model, losses = train(E, x, y, ctx=trie.ctx, epochs=epochs)
    info = evaluate(E, model, prof)
    info["train_rows"] = int(len(x))
    info["final_loss"] = float(np.mean(losses[-20:])) if losses else None
    info["query"] = query
    return model, info, prof
