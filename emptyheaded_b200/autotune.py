"""Schedule autotuner for the COUNT kernels.

Picks, for one trie and one layout assignment, the schedule knobs of
eh_exec_config by timing the intersection kernel on the device (CUDA events
inside the engine, eh_query_stats.kernel_ms):

  warps        warps per block of the persistent kernel
  smem_words   shared staging per warp (u32 words): the tile width a staged
               N(b) may have before it is probed in global memory
  chunk        probes per work item (work-chunk size of the queue)
  long_row     size-class boundary: rows with at least this many candidates
               run warp-wide, shorter rows are flattened over the lanes

Coordinate descent from the measured defaults: each knob is swept with the
others fixed, the best value kept, two rounds.  Every timed run's count is
checked against the first one, so tuning can never change a result.
"""
import statistics

GRID = {
    "smem_words": (512, 1024, 1536),
    "chunk": (16384, 32768, 65536, 131072),
    "long_row": (16, 32, 64, 128),
    "warps": (4, 8, 16),
}
DEFAULT = {"warps": 8, "smem_words": 1024, "chunk": 32768, "long_row": 32}


def _time(trie, cfg, query, reps, want):
    ks = []
    for _ in range(reps):
        c, st = trie.count(query, stats=True, config=cfg)
        if want is not None and c != want:
            raise AssertionError("schedule changed the count: %d != %d" % (c, want))
        ks.append(st["kernel_ms"])
    return statistics.median(ks)


def tune(trie, query="triangle", reps=3, rounds=2, grid=None):
    """Returns (best config dict, log of (config, kernel_ms))."""
    grid = grid or GRID
    want = trie.count(query, config=DEFAULT)
    best = dict(DEFAULT)
    best_t = _time(trie, best, query, reps, want)
    log = [(dict(best), best_t)]
    for _ in range(rounds):
        improved = False
        for knob, values in grid.items():
            for v in values:
                if v == best[knob]:
                    continue
                cfg = dict(best)
                cfg[knob] = v
                t = _time(trie, cfg, query, reps, want)
                log.append((cfg, t))
                if t < best_t * 0.99:
                    best, best_t, improved = cfg, t, True
        if not improved:
            break
    return best, log
