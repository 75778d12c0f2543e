"""Search benchmark: plain BM25 Search on a resident 10M-doc index, bit-exact top-K.

Workload (one "step" = one Search of one query batch): seeded synthetic corpus of
10,000,000 documents, vocabulary 1,000,000 with Zipf(1.1) token ranks, lognormal
lengths with mean 60 (sigma 0.5), k1 1.5, b 0.75, eager FP32 posting scores in
CSC resident in HBM; batches of 8 queries x 3 distinct terms drawn by document
frequency, K = 10; two batches A/B alternate as in the reference's benchmark.

  value   queries/s of the device-resident Search (inputs already in HBM), timed
          per step with CUDA events on the launching stream, L2 flushed between
          steps (a 256 MiB write), summed over the K timed steps; max over ranks.
  e2e     queries/s of the public C-ABI call bm25_search with host buffers
          (pack, graph replay with H2D + kernel + D2H, synchronise, validate),
          host wall-clock per call, L2 flushed between calls.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

  learned_pruned   the same Searches with learned starting bounds: a threshold MLP
          (32 -> 64 -> 64 -> 1) trained on the GPU by the engine's own kernels on
          200k generated queries of the same shape (targets: the plain engine's
          K-th scores), then timed as above (device-resident and through
          bm25_search_learned), beside the safe bounds alone; every result checked
          bit for bit against the oracle.
  tuning  before the timed region, the session's runtime knobs (warp-tile claim
          size and tail claims) are timed on a sample batch of its own seed and
          the fastest kept (autotune.tune; every setting bit-checked against the
          first); the mix and block-max legs tune their learned routing cut the
          same way.  --no-tune keeps the defaults of the plain leg.
  batched_mix, blockmax_c4, reference_shape, serving, cpu_baseline_bm25s: the
          C3, C4, reference-shaped, C5 and bm25s legs (see their functions).

--impl reference times the reference's own CPU search (oracle/_ref, compiled from
the reference's sources; the oracle's C restatement where that was not built) on
the same corpus and batches with every host thread.
"""

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'Search QPS + p50/p95 ms, 10M docs K10: plain vs learned-pruned, bit-exact top-K'
UNIT = 'queries/s'
WORKLOAD = 'synthetic_10m'
Q, TERMS, K = 8, 3, 10
SEED_A, SEED_B = 20261014, 20261015
FALLBACK_HBM_GBS = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def percentile(values, p):
    v = sorted(values)
    return v[min(len(v) - 1, max(0, int(round(p / 100.0 * (len(v) - 1)))))]


def hbm_peak():
    path = ROOT / 'MEASURED_PEAKS.json'
    try:
        peaks = json.loads(path.read_text())
        return float(peaks['hbm_gbs']), 'measured'
    except Exception:
        return FALLBACK_HBM_GBS, 'fallback'


def algorithmic_bytes(df, vocab, offsets, words, k, distinct=False):
    """Posting bytes the Search must read: per in-vocabulary query word df*8 (int32 id + f32 score)
    + 16 B of indptr, plus the Q*K*8 B result.  Every query's words count (a word shared by several
    queries counts once per query) unless `distinct`: the tile-major kernel reads a shared word's
    postings from DRAM once and from L2 for the other queries, so DRAM traffic follows the distinct
    figure."""
    seq = set(int(x) for x in words) if distinct else words
    total = 0
    for w in seq:
        if 0 <= w < vocab:
            total += int(df[w]) * 8 + 16
    return total + (offsets.size - 1) * k * 8


def traffic_from_profile(name='tile_group_kernel_synthetic_10m.txt'):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = ROOT / 'profiles' / name
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.startswith('traffic_bytes_per_launch:'):
            try:
                return float(line.split(':', 1)[1].split()[0])
            except ValueError:
                return None
    return None


class Clocks:
    """nvidia-smi sampler for the timed region."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        self.path = tempfile.NamedTemporaryFile(prefix='clocks_', suffix='.csv', delete=False).name
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', f'--id={self.device}', f'--query-gpu={self.FIELDS}', '--format=csv,noheader,nounits',
                 '-lms', '200'], stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(',')]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == 'active'})
        return {'sm_mhz': statistics.median(sm) if sm else None,
                'sm_max_mhz': float(rows[0][2]) if rows[0][2].replace('.', '').isdigit() else None,
                'reasons': reasons, 'samples': len(rows)}


def setup_dist(gpus):
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world != gpus:
        log(f'warning: --gpus {gpus} but WORLD_SIZE {world}')
    return rank, world, local


def build_corpus(pkg, docs=0, vocab=0):
    import dataclasses
    spec = pkg.CONFIG_SHAPES[WORKLOAD]
    if docs or vocab:  # reduced copies of the workload, for ncu captures that must stay small
        spec = dataclasses.replace(spec, docs=docs or spec.docs, vocab=vocab or spec.vocab)
    t = time.perf_counter()
    index = pkg.synthetic_index(spec)
    log(f'corpus: N={index.num_docs} V={index.vocab} M={index.postings} in {time.perf_counter() - t:.1f}s')
    return spec, index


def batches(pkg, index, rank):
    a = pkg.synthetic_queries(index.offsets, Q, TERMS, TERMS, SEED_A + 1000 * rank)
    b = pkg.synthetic_queries(index.offsets, Q, TERMS, TERMS, SEED_B + 1000 * rank)
    return [a, b]


def cpu_search_leg(index, sets, k, budget_s, max_steps, warmup=1):
    """The reference's CPU search (oracle/_ref) or the oracle's restatement, all host threads."""
    from oracle import oracle
    threads = os.cpu_count() or 1
    if oracle.reference_available():
        session = oracle.ReferenceCpuSession(index, k, threads, shards=threads, query_capacity=Q,
                                             word_capacity=Q * TERMS)

        def run(i):
            return session.search(*sets[i % 2])[:2]

        kind, cores = 'reference', session.threads
        note = ('reference bm25cpu::CpuSearchSession (cpu_index_search.h) compiled from its sources; '
                'its contribution uses the hard-coded k1=1.2 (2.2F) on the same postings, same work')
    else:
        data = oracle.contributions(index, 1.5)

        def run(i):
            return oracle.search(index.offsets, index.docs, data, index.num_docs, *sets[i % 2], k, threads=threads)

        kind, cores = 'port', min(threads, Q)
        note = 'oracle C restatement (term-order scatter + bounded heap), OpenMP over queries'
    for i in range(warmup):
        run(i)
    times = []
    t_start = time.perf_counter()
    i = 0
    while i < max_steps and (time.perf_counter() - t_start) < budget_s:
        t0 = time.perf_counter()
        run(i)
        times.append(time.perf_counter() - t0)
        i += 1
    total = sum(times)
    return {'value': Q * len(times) / total, 'unit': UNIT, 'cores': cores, 'kind': kind,
            'sample': f'{len(times)} full Searches of {Q} queries x {TERMS} terms (A/B alternating) on the same '
                      f'10M-doc corpus; {note}',
            'p50_ms': percentile(times, 50) * 1e3, 'p95_ms': percentile(times, 95) * 1e3}


class StepCheck:
    """Bit-checks every timed Search of a leg, as the reference's Measure compares every timed result
    with its checkpoint (FR/test/ascendhost/bm25/benchmark_common.h:70-95).  After each timed step,
    outside its timed interval, the step's device outputs are copied into a slot of their own; after
    the timed loop every slot is compared bit for bit with the expected outputs of that step's batch
    (the oracle's on rank 0, where they were computed).  `outputs`: the device tensors a step writes;
    `expected(i)`: the list of host arrays step i must equal (None: not checked); `length`: how many
    leading elements of each output a step writes (packed batches)."""

    def __init__(self, outputs, expected, steps, length=None):
        import torch
        self.outputs = outputs
        self.expected = expected
        self.length = length
        self.slots = [[torch.empty_like(t) for t in outputs] for _ in range(steps)]
        self.checked = 0
        self.mismatched = 0

    def capture(self, i):
        for dst, src in zip(self.slots[i], self.outputs):
            dst.copy_(src)

    def verify(self, n):
        for i in range(n):
            want = self.expected(i)
            if want is None:
                continue
            m = self.length(i) if self.length else None
            ok = True
            for got, w in zip(self.slots[i], want):
                g = got.reshape(-1)[:m].cpu().numpy() if m is not None else got.cpu().numpy()
                w = np.asarray(w).reshape(-1)[:g.size] if m is not None else np.asarray(w)
                ok &= bool(np.array_equal(g.reshape(-1).view(np.uint32), w.reshape(-1).view(np.uint32)))
            self.checked += 1
            self.mismatched += 0 if ok else 1

    def report(self):
        return {'checked_searches': self.checked, 'mismatched': self.mismatched,
                'bit_exact': self.checked > 0 and self.mismatched == 0}


def cpu_bm25s_leg(index, k1, sets, want, budget_s=6.0, max_steps=20):
    """bm25s's native retrieve (numba; oracle/bm25s_port.py restates its query step) on the same corpus
    and batches, timed at n_threads in {1, 8, all host threads}: the reference's second CPU baseline
    (standalone/bm25s_benchmark.py:76-95).  Its ranking keeps bm25s's non-strict ties, so its results
    are checked against the oracle's as sorted score lists."""
    from oracle import bm25s_port, oracle
    if not bm25s_port.available():
        return {'unavailable': 'numba is not installed'}
    data = oracle.contributions(index, k1)
    cores = os.cpu_count() or 1
    out = {'kind': 'port', 'what': 'bm25s native retrieve (pinned 03eac5a8) restated with numba: zeros(N), '
                                   'term-order scatter-add, size-K heap, sorted', 'cores': cores, 'threads': {}}
    for n_threads in sorted({1, min(8, cores), cores}):
        bm25s_port.retrieve(index.offsets, index.docs, data, index.num_docs, *sets[0], K, n_threads)  # compiles
        times, ok = [], True
        t_start = time.perf_counter()
        i = 0
        while i < max_steps and time.perf_counter() - t_start < budget_s:
            t0 = time.perf_counter()
            bs, _ = bm25s_port.retrieve(index.offsets, index.docs, data, index.num_docs, *sets[i % 2], K, n_threads)
            times.append(time.perf_counter() - t0)
            if want is not None:
                ok &= bool(np.array_equal(np.sort(bs, axis=1), np.sort(want[i % 2][0], axis=1)))
            i += 1
        out['threads'][str(n_threads)] = {'value': Q * len(times) / sum(times), 'unit': UNIT,
                                          'p50_ms': percentile(times, 50) * 1e3, 'searches': len(times),
                                          'scores_match_oracle': ok}
    best = max(out['threads'].values(), key=lambda r: r['value'])
    out['value'] = best['value']
    out['unit'] = UNIT
    return out


def timed_device(session, step, steps, warmup, flush, stream, world, with_clocks=None, check=None):
    """Device-resident steps timed with CUDA events on the launching stream, L2 flushed between
    steps; returns (step ms, main-kernel ms, clocks).

    Two passes over the same K steps.  The first gives the step times and the clocks: only the
    step's own events are recorded.  The second also has the engine record an event pair around
    its main kernel, for that kernel's duration; an event between two kernels keeps the later one
    from starting while the earlier one runs (programmatic dependent launch), so the second pass
    is slower and gives no step times.  The engine's counters are those of the second pass."""
    import torch
    import torch.distributed as dist

    def run(marks):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        session.kernel_timing(marks)
        session.search_stats(reset=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        if with_clocks and not marks:
            with_clocks.start()
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            step(i)
            ends[i].record(stream)
            if check is not None:
                check.capture(i)  # after the step's end event: not in its timed interval
        torch.cuda.synchronize()
        if check is not None:
            check.verify(steps)
        clocks = with_clocks.stop() if with_clocks and not marks else None
        status = session.device_status()
        if status != 0:
            raise RuntimeError(f'device status {status:#x} set during the timed region')
        kernel = [float(x) for x in session.kernel_times()] if marks else None
        session.kernel_timing(False)
        return [a.elapsed_time(b) for a, b in zip(starts, ends)], kernel, clocks

    with torch.cuda.stream(stream):
        for i in range(warmup):
            step(i)
        stream.synchronize()
        status = session.device_status()
        if status != 0:
            raise RuntimeError(f'device status {status:#x} set during warm-up')
        step_ms, _, clock_info = run(False)
        _, kernel_ms, _ = run(True)
    if len(kernel_ms) != steps:
        raise RuntimeError(f'{len(kernel_ms)} kernel timings for {steps} steps')
    return step_ms, kernel_ms, clock_info


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device='cuda', dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def learned_leg(pkg, args, spec, index, session, sets, want, flush, stream, dev_sets, local, world):
    """Learned-pruned Search on the same session, batches and timing rules as the plain line.

    A threshold MLP is trained on the GPU (the engine's own kernels) from queries of the same
    shape whose targets the plain engine computes, then the learned Search is timed device-resident
    and end to end; the safe bounds alone (the method without the network) are timed beside it."""
    import torch
    t = time.perf_counter()
    cap = 2048
    trainer = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=cap, word_capacity=cap * TERMS, max_k=K, device_id=local,
                                        prune=True)
    model = pkg.learned.fit(trainer, index.offsets, queries=args.train_queries, ks=(K,), lo=TERMS, hi=TERMS,
                            seed=args.train_seed, steps=args.train_steps, batch=4096, gen_batch=cap,
                            target_fallback=args.target_fallback, device=f'cuda:{local}')
    trainer.close()
    train_s = time.perf_counter() - t
    log(f'threshold model trained in {train_s:.1f}s: {model.report}')
    d_scores = torch.empty((Q, K), dtype=torch.float32, device='cuda')
    d_ids = torch.empty((Q, K), dtype=torch.int32, device='cuda')
    d_exact = torch.empty(Q, dtype=torch.int32, device='cuda')

    def step(i):
        o, w = dev_sets[i % 2]
        session.search_learned_device(o.data_ptr(), w.data_ptr(), Q, K, d_scores.data_ptr(), d_ids.data_ptr(),
                                      d_exact.data_ptr(), stream.cuda_stream)

    out = {}
    for label, m in (('safe_bounds_only', None), ('learned', model)):
        session.set_threshold_model(m)
        parity = True
        if want is not None:
            for qs, (rs, ri) in zip(sets, want):
                gs, gi, _ = session.search_learned(qs, K)
                parity &= bool(np.array_equal(gi, ri) and np.array_equal(gs.view(np.uint32), rs.view(np.uint32)))
        check = StepCheck([d_scores, d_ids], lambda i: want[i % 2] if want is not None else None, args.steps)
        step_ms, kernel_ms, _ = timed_device(session, step, args.steps, args.warmup, flush, stream, world, check=check)
        stats = session.search_stats(reset=True)
        total = max_over_ranks(sum(step_ms), world)
        host_ms, fallbacks, e2e_checked, e2e_bad = [], 0, 0, 0
        lout = (np.empty((Q, K), np.float32), np.empty((Q, K), np.int32), np.empty(Q, np.int32))
        for i in range(args.warmup):
            session.search_learned(sets[i % 2], K, out=lout)
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            gs, gi, exact = session.search_learned(sets[i % 2], K, out=lout)
            host_ms.append((time.perf_counter() - t0) * 1e3)
            fallbacks += int(np.sum(exact == 0))
            if want is not None:
                e2e_checked += 1
                e2e_bad += 0 if same_bits((gs, gi), want[i % 2]) else 1
        e2e_total = max_over_ranks(sum(host_ms), world)
        out[label] = {
            'value': world * Q * args.steps / (total / 1e3), 'unit': UNIT,
            'p50_ms': percentile(step_ms, 50), 'p95_ms': percentile(step_ms, 95),
            'pruned_kernel_ms_avg': sum(kernel_ms) / len(kernel_ms),
            'e2e': {'value': world * Q * args.steps / (e2e_total / 1e3), 'unit': UNIT,
                    'p50_ms': percentile(host_ms, 50), 'p95_ms': percentile(host_ms, 95),
                    'path': 'bm25_search_learned (C ABI, host buffers): one graph replay'},
            'fallback_share': fallbacks / (Q * args.steps),
            # learned bounds, plan, block bound, block score, final select, then the retry pass's block
            # bound, block score and final select (an empty list ends them at once)
            'gpu_launches': args.steps * 8,
            'per_search': {key: v / args.steps for key, v in stats.items()},
            'bit_exact_vs_oracle': parity if want is not None else None,
            'timed_parity': dict(check.report(), e2e_checked=e2e_checked, e2e_mismatched=e2e_bad),
        }
    out['learned']['model'] = {'train_queries': model.report['train_queries'], 'train_s': train_s,
                               'margin': model.margin, 'val_fallback': model.report['val_fallback'],
                               'first_loss': model.report['first_loss'], 'last_loss': model.report['last_loss'],
                               'trained_with': 'bm25_mlp_gradient + bm25_mlp_adam (engine kernels)'}
    return out


MIX_WORKLOAD = 'passages_8p8m'
MIX_Q, MIX_TERMS, MIX_KS = 256, (2, 12), (10, 100, 1000)


def mix_leg(pkg, args, local, world, flush, stream, rank):
    """The batched mix: 8.8M passages (V 2.5M, Zipf 1.05, mean 56), 256 queries per Search with
    2-12 terms drawn by df and K drawn from {10, 100, 1000} per query, all in one Search
    (bm25_search_batch: one graph replay).  Plain and learned-pruned, device-resident and e2e."""
    import torch
    spec = pkg.CONFIG_SHAPES[MIX_WORKLOAD]
    t = time.perf_counter()
    index = pkg.synthetic_index(spec)
    log(f'mix corpus: N={index.num_docs} V={index.vocab} M={index.postings} in {time.perf_counter() - t:.1f}s')
    lo, hi = MIX_TERMS
    batches = []
    for b in range(2):
        qo, w = pkg.synthetic_queries(index.offsets, MIX_Q, lo, hi, 880000 + 1000 * rank + b)
        ks = np.random.default_rng(770 + 1000 * rank + b).choice(MIX_KS, MIX_Q).astype(np.int32)
        batches.append((qo, w, ks))
    kmax = max(MIX_KS)
    session = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=MIX_Q, word_capacity=MIX_Q * hi, max_k=kmax,
                                        device_id=local, prune=True)
    parity = None
    expected = None
    if rank == 0:
        from oracle import oracle
        data = oracle.contributions(index, spec.k1)
        expected = [oracle_packed(index, data, qo, w, ks, MIX_KS) for qo, w, ks in batches]
        del data
        ok = all(same_bits(session.search_batch((qo, w), ks)[:2], want)
                 for (qo, w, ks), want in zip(batches, expected))
        parity = {'batches': len(batches), 'queries_checked': MIX_Q * len(batches), 'bit_exact': ok,
                  'against': 'oracle (C restatement), per K group'}
        log(f'mix parity vs oracle: {parity}')
    t = time.perf_counter()
    cap = 1024
    trainer = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=cap, word_capacity=cap * hi, max_k=kmax, device_id=local,
                                        prune=True)
    model = pkg.learned.fit(trainer, index.offsets, queries=args.mix_train_queries, ks=MIX_KS, lo=lo, hi=hi,
                            seed=args.train_seed, steps=args.train_steps, batch=4096, gen_batch=cap,
                            target_fallback=args.target_fallback, device=f'cuda:{local}')
    trainer.close()
    train_s = time.perf_counter() - t
    log(f'mix threshold model trained in {train_s:.1f}s: {model.report}')
    dev = []
    for qo, w, ks in batches:
        koff = np.zeros(MIX_Q + 1, np.int64)
        np.cumsum(ks, out=koff[1:])
        dev.append(tuple(torch.from_numpy(x).cuda() for x in (qo, w, ks, koff[:-1].copy())))
    d_s = torch.empty(MIX_Q * kmax, dtype=torch.float32, device='cuda')
    d_i = torch.empty(MIX_Q * kmax, dtype=torch.int32, device='cuda')
    d_x = torch.empty(MIX_Q, dtype=torch.int32, device='cuda')
    out = {'workload': MIX_WORKLOAD, 'docs': spec.docs, 'vocab': spec.vocab, 'zipf_s': spec.zipf_s,
           'len_mean': spec.len_mean, 'postings': index.postings, 'queries_per_search': MIX_Q,
           'terms': f'U{{{lo}..{hi}}} drawn by df', 'k': 'per query from {10, 100, 1000}', 'parity': parity,
           'model': {'train_queries': model.report['train_queries'], 'train_s': train_s, 'margin': model.margin,
                     'val_fallback': model.report['val_fallback']}}
    steps = max(3, args.steps // 4)
    totals = [int(ks.sum()) for _, _, ks in batches]
    sample_qo, sample_w = pkg.synthetic_queries(index.offsets, MIX_Q, lo, hi, 880077 + 1000 * rank)
    sample_ks = np.random.default_rng(777 + 1000 * rank).choice(MIX_KS, MIX_Q).astype(np.int32)
    out['tuning'] = route_tuning(pkg, session, model, (sample_qo, sample_w, sample_ks), kmax)
    log(f"mix tuning: {out['tuning']}")
    for label, learned in (('plain', False), ('learned', True)):
        session.set_threshold_model(model if learned else None)

        def step(i):
            o, w, k, ko = dev[i % 2]
            session.search_batch_device(o.data_ptr(), w.data_ptr(), k.data_ptr(), ko.data_ptr(), MIX_Q, kmax,
                                        d_s.data_ptr(), d_i.data_ptr(), d_x.data_ptr(), learned,
                                        stream.cuda_stream)

        check = StepCheck([d_s, d_i], lambda i: expected[i % 2] if expected else None, steps,
                          length=lambda i: totals[i % 2])
        step_ms, kernel_ms, _ = timed_device(session, step, steps, args.warmup, flush, stream, world, check=check)
        stats = session.search_stats(reset=True)
        total = max_over_ranks(sum(step_ms), world)
        host_ms, fallbacks, e2e_checked, e2e_bad = [], 0, 0, 0
        for i in range(args.warmup):
            session.search_batch(batches[i % 2][:2], batches[i % 2][2], learned=learned)
        for i in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = session.search_batch(batches[i % 2][:2], batches[i % 2][2], learned=learned)
            host_ms.append((time.perf_counter() - t0) * 1e3)
            if learned:
                fallbacks += int(np.sum(r[3] == 0))
            if expected:
                e2e_checked += 1
                e2e_bad += 0 if same_bits(r[:2], expected[i % 2]) else 1
        e2e_total = max_over_ranks(sum(host_ms), world)
        out[label] = {'value': world * MIX_Q * steps / (total / 1e3), 'unit': UNIT,
                      'p50_ms': percentile(step_ms, 50), 'p95_ms': percentile(step_ms, 95),
                      'main_kernel_ms_avg': sum(kernel_ms) / len(kernel_ms),
                      'e2e': {'value': world * MIX_Q * steps / (e2e_total / 1e3), 'unit': UNIT,
                              'p50_ms': percentile(host_ms, 50), 'p95_ms': percentile(host_ms, 95)},
                      'per_search': {key: v / steps for key, v in stats.items()}, 'steps': steps,
                      'timed_parity': dict(check.report(), e2e_checked=e2e_checked, e2e_mismatched=e2e_bad)}
        if learned:
            out[label]['fallback_share'] = fallbacks / (MIX_Q * steps)
    out['speedup_learned_vs_plain'] = out['learned']['value'] / out['plain']['value']
    out['e2e_speedup_learned_vs_plain'] = out['learned']['e2e']['value'] / out['plain']['e2e']['value']
    session.close()
    return out


BLOCKMAX_WORKLOAD = 'blockmax_4p2m'
BLOCKMAX_Q, BLOCKMAX_TERMS, BLOCKMAX_KS, BLOCKMAX_EVAL = 250, (2, 10), (10, 100), 10_000


def oracle_packed(index, data, qo, w, ks, kset):
    """The oracle's results of a batch with a K per query, packed by query as bm25_search_batch packs
    them (query i's ks[i] entries start at ks[0] + ... + ks[i-1]); one oracle call per K."""
    from oracle import oracle
    koff = np.zeros(ks.size + 1, np.int64)
    np.cumsum(ks, out=koff[1:])
    ps = np.empty(int(koff[-1]), np.float32)
    pi = np.empty(int(koff[-1]), np.int32)
    for k in kset:
        sel = np.nonzero(ks == k)[0]
        if sel.size == 0:
            continue
        rows = [w[qo[i]:qo[i + 1]] for i in sel]
        o = np.zeros(len(rows) + 1, np.int64)
        o[1:] = np.cumsum([len(r) for r in rows])
        rs, ri = oracle.search(index.offsets, index.docs, data, index.num_docs, o,
                               np.concatenate(rows).astype(np.int32), int(k), threads=os.cpu_count() or 1)
        for j, i in enumerate(sel):
            ps[koff[i]:koff[i + 1]] = rs[j]
            pi[koff[i]:koff[i + 1]] = ri[j]
    return ps, pi


ROUTE_CUTS = (0.3, 0.45, 0.6, 0.8, 1.0)


def route_tuning(pkg, session, model, sample, kmax):
    """The learned routing cut (share of a query's blocks kept above which the query is streamed;
    1.0: none is), timed on a sample batch with a K per query (its own seed, not a timed batch),
    every cut bit-checked against the first; the fastest is kept on the session."""
    t = time.perf_counter()
    session.set_threshold_model(model)
    qo, w, ks = sample
    best, table = pkg.autotune.tune(session, (qo, w), kmax, space={'prune_route': ROUTE_CUTS}, learned=True,
                                    ks=ks, reps=5)
    return {'chosen': {'prune_route': best['prune_route']}, 'ms': {str(c['prune_route']): round(ms, 4)
                                                                   for c, ms in table},
            'sample': f'one batch of {qo.size - 1} queries (its own seed), 5 timed Searches per cut',
            'seconds': round(time.perf_counter() - t, 2)}


def same_bits(got, want):
    """(scores, ids) pairs equal bit for bit."""
    return all(np.array_equal(np.asarray(g).reshape(-1).view(np.uint32), np.asarray(x).reshape(-1).view(np.uint32))
               for g, x in zip(got, want))


def split_queries(qoffsets, words, ks, per_search):
    """Packed queries (offsets [Q+1], words) with a K each, cut into Searches of per_search queries
    (the last one shorter when Q is not a multiple): a list of (offsets from 0, words, ks)."""
    out = []
    for a0 in range(0, qoffsets.size - 1, per_search):
        a1 = min(a0 + per_search, qoffsets.size - 1)
        out.append(((qoffsets[a0:a1 + 1] - qoffsets[a0]).astype(np.int64),
                    words[qoffsets[a0]:qoffsets[a1]].copy(), ks[a0:a1].copy()))
    return out


def blockmax_leg(pkg, args, local, world, flush, stream, rank):
    """The block-max workload: 4.2M docs (V 1M, mean length 80), a threshold model trained on
    200k queries, then 10k held-out queries of 2-10 terms drawn by df with K drawn from {10, 100}
    per query, answered 250 to a Search (40 Searches, one pass over the set per timed pass), plain
    and learned-pruned.  Besides queries/s: the postings each Search touches either way."""
    import torch
    spec = pkg.CONFIG_SHAPES[BLOCKMAX_WORKLOAD]
    t = time.perf_counter()
    index = pkg.synthetic_index(spec)
    log(f'block-max corpus: N={index.num_docs} V={index.vocab} M={index.postings} in {time.perf_counter() - t:.1f}s')
    lo, hi = BLOCKMAX_TERMS
    qo_all, w_all = pkg.synthetic_queries(index.offsets, BLOCKMAX_EVAL, lo, hi, 440000 + 1000 * rank)
    ks_all = np.random.default_rng(550 + 1000 * rank).choice(BLOCKMAX_KS, BLOCKMAX_EVAL).astype(np.int32)
    batches = split_queries(qo_all, w_all, ks_all, BLOCKMAX_Q)
    n_batches = len(batches)
    kmax = max(BLOCKMAX_KS)
    session = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=BLOCKMAX_Q, word_capacity=BLOCKMAX_Q * hi, max_k=kmax,
                                        device_id=local, prune=True)
    parity = None
    expected = None
    if rank == 0:
        from oracle import oracle
        t = time.perf_counter()
        data = oracle.contributions(index, spec.k1)
        expected = [oracle_packed(index, data, qo, w, ks, BLOCKMAX_KS) for qo, w, ks in batches]
        del data
        ok = all(same_bits(session.search_batch((qo, w), ks)[:2], want)
                 for (qo, w, ks), want in zip(batches, expected))
        parity = {'batches': n_batches, 'c4_queries_checked': BLOCKMAX_EVAL, 'bit_exact': ok,
                  'against': 'oracle (C restatement), per K group', 'oracle_s': time.perf_counter() - t}
        log(f'block-max parity vs oracle: {parity}')
    t = time.perf_counter()
    cap = 1024
    trainer = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=cap, word_capacity=cap * hi, max_k=kmax, device_id=local,
                                        prune=True)
    model = pkg.learned.fit(trainer, index.offsets, queries=args.blockmax_train_queries, ks=BLOCKMAX_KS, lo=lo,
                            hi=hi, seed=args.train_seed, steps=args.train_steps, batch=4096, gen_batch=cap,
                            target_fallback=args.target_fallback, device=f'cuda:{local}')
    trainer.close()
    train_s = time.perf_counter() - t
    log(f'block-max threshold model trained in {train_s:.1f}s: {model.report}')
    dev = []
    for qo, w, ks in batches:
        koff = np.zeros(BLOCKMAX_Q + 1, np.int64)
        np.cumsum(ks, out=koff[1:])
        dev.append(tuple(torch.from_numpy(x).cuda() for x in (qo, w, ks, koff[:-1].copy())))
    d_s = torch.empty(BLOCKMAX_Q * kmax, dtype=torch.float32, device='cuda')
    d_i = torch.empty(BLOCKMAX_Q * kmax, dtype=torch.int32, device='cuda')
    d_x = torch.empty(BLOCKMAX_Q, dtype=torch.int32, device='cuda')
    out = {'workload': BLOCKMAX_WORKLOAD, 'docs': spec.docs, 'vocab': spec.vocab, 'len_mean': spec.len_mean,
           'postings': index.postings, 'eval_queries': BLOCKMAX_EVAL, 'queries_per_search': BLOCKMAX_Q,
           'terms': f'U{{{lo}..{hi}}} drawn by df', 'k': 'per query from {10, 100}', 'parity': parity,
           'model': {'train_queries': model.report['train_queries'], 'train_s': train_s, 'margin': model.margin,
                     'val_fallback': model.report['val_fallback']}}
    steps = n_batches  # one pass over the held-out set
    totals = [int(ks.sum()) for _, _, ks in batches]
    sample_qo, sample_w = pkg.synthetic_queries(index.offsets, BLOCKMAX_Q, lo, hi, 420077 + 1000 * rank)
    sample_ks = np.random.default_rng(477 + 1000 * rank).choice(BLOCKMAX_KS, BLOCKMAX_Q).astype(np.int32)
    out['tuning'] = route_tuning(pkg, session, model, (sample_qo, sample_w, sample_ks), kmax)
    log(f"block-max tuning: {out['tuning']}")
    for label, learned in (('plain', False), ('learned', True)):
        session.set_threshold_model(model if learned else None)

        def step(i):
            o, w, k, ko = dev[i % n_batches]
            session.search_batch_device(o.data_ptr(), w.data_ptr(), k.data_ptr(), ko.data_ptr(), BLOCKMAX_Q, kmax,
                                        d_s.data_ptr(), d_i.data_ptr(), d_x.data_ptr(), learned,
                                        stream.cuda_stream)

        check = StepCheck([d_s, d_i], lambda i: expected[i % n_batches] if expected else None, steps,
                          length=lambda i: totals[i % n_batches])
        step_ms, kernel_ms, _ = timed_device(session, step, steps, args.warmup, flush, stream, world, check=check)
        stats = session.search_stats(reset=True)
        total = max_over_ranks(sum(step_ms), world)
        host_ms, fallbacks, e2e_checked, e2e_bad = [], 0, 0, 0
        for i in range(args.warmup):
            session.search_batch(batches[i % n_batches][:2], batches[i % n_batches][2], learned=learned)
        for i in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = session.search_batch(batches[i][:2], batches[i][2], learned=learned)
            host_ms.append((time.perf_counter() - t0) * 1e3)
            if learned:
                fallbacks += int(np.sum(r[3] == 0))
            if expected:
                e2e_checked += 1
                e2e_bad += 0 if same_bits(r[:2], expected[i]) else 1
        e2e_total = max_over_ranks(sum(host_ms), world)
        per = {key: v / steps for key, v in stats.items()}
        out[label] = {'value': world * BLOCKMAX_Q * steps / (total / 1e3), 'unit': UNIT,
                      'p50_ms': percentile(step_ms, 50), 'p95_ms': percentile(step_ms, 95),
                      'main_kernel_ms_avg': sum(kernel_ms) / len(kernel_ms),
                      'e2e': {'value': world * BLOCKMAX_Q * steps / (e2e_total / 1e3), 'unit': UNIT,
                              'p50_ms': percentile(host_ms, 50), 'p95_ms': percentile(host_ms, 95)},
                      'per_search': per, 'steps': steps,
                      'timed_parity': dict(check.report(), e2e_checked=e2e_checked, e2e_mismatched=e2e_bad),
                      # postings read block by block plus postings streamed whole (8 B each)
                      'posting_bytes_per_search': 8.0 * (per['postings_read'] + per['postings_copied'])}
        if learned:
            out[label]['fallback_share'] = fallbacks / BLOCKMAX_EVAL
    out['speedup_learned_vs_plain'] = out['learned']['value'] / out['plain']['value']
    out['e2e_speedup_learned_vs_plain'] = out['learned']['e2e']['value'] / out['plain']['e2e']['value']
    out['posting_bytes_learned_vs_plain'] = (out['learned']['posting_bytes_per_search'] /
                                             max(out['plain']['posting_bytes_per_search'], 1.0))
    session.close()
    return out


REFSHAPE_WORKLOAD = 'reference_10m'
A5_PUBLISHED_MS = {'A': 1.759, 'B': 1.742}  # reference Search medians at 10M docs on its own corpus (docs/BM25S_PERFORMANCE.md:32)


def refshape_leg(pkg, args, local, world, flush, stream, rank):
    """The reference's own benchmark corpus shape at 10M documents (uniform over 1024 terms, lengths
    16..48, seed 20261014, k1 1.2, b 0.75; generated by this repo's seeded generator, the same shape
    as standalone/large_corpus.py:58-62) with the reference's query sets A and B (fixtures/A.txt,
    B.txt, committed in tests/golden/large_corpus_n2048.npz): the plain Search timed device-resident
    and end to end like the headline line, every timed result checked against the oracle, beside the
    reference's published median on this shape and, on rank 0, its own C++ CPU search on this box."""
    import torch
    spec = pkg.CONFIG_SHAPES[REFSHAPE_WORKLOAD]
    t = time.perf_counter()
    index = pkg.synthetic_index(spec)
    log(f'reference-shaped corpus: N={index.num_docs} V={index.vocab} M={index.postings} in '
        f'{time.perf_counter() - t:.1f}s')
    fx = np.load(ROOT / 'tests' / 'golden' / 'large_corpus_n2048.npz')
    sets = [(fx['A_offsets'].astype(np.int64), fx['A_words'].astype(np.int32)),
            (fx['B_offsets'].astype(np.int64), fx['B_words'].astype(np.int32))]
    q = sets[0][0].size - 1
    session = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=q, word_capacity=int(sets[0][0][-1]), max_k=K,
                                        device_id=local)
    want = None
    out = {'workload': REFSHAPE_WORKLOAD, 'docs': spec.docs, 'vocab': spec.vocab, 'postings': index.postings,
           'lengths': 'uniform 16..48', 'queries': f'the reference\'s sets A and B ({q} x 3 words)', 'k': K,
           'k1': spec.k1, 'b': spec.b, 'a5_published_median_ms': A5_PUBLISHED_MS}
    if rank == 0:
        from oracle import oracle
        data = oracle.contributions(index, spec.k1)
        want = [oracle.search(index.offsets, index.docs, data, index.num_docs, *qs, K) for qs in sets]
        del data
        out['parity'] = {'bit_exact': all(same_bits(session.search(qs, K), w) for qs, w in zip(sets, want)),
                         'against': 'oracle (C restatement)'}
        if oracle.reference_available():  # k1 = 1.2: the reference's own search gives the same bits
            ref = oracle.ReferenceCpuSession(index, K, os.cpu_count() or 1, query_capacity=q,
                                             word_capacity=int(sets[0][0][-1]))
            ref_ms, ref_ok = [], True
            for i in range(min(20, args.steps)):
                t0 = time.perf_counter()
                rs, ri, _ = ref.search(*sets[i % 2])
                ref_ms.append((time.perf_counter() - t0) * 1e3)
                ref_ok &= same_bits((rs, ri), want[i % 2])
            out['reference_cpu'] = {'p50_ms': percentile(ref_ms, 50), 'queries_per_s': q * len(ref_ms) / (sum(ref_ms) / 1e3),
                                    'threads': ref.threads, 'same_bits_as_oracle': bool(ref_ok),
                                    'what': 'bm25cpu::CpuSearchSession compiled from the reference sources'}
    dev = [(torch.from_numpy(o).cuda(), torch.from_numpy(w).cuda()) for o, w in sets]
    d_s = torch.empty((q, K), dtype=torch.float32, device='cuda')
    d_i = torch.empty((q, K), dtype=torch.int32, device='cuda')

    def step(i):
        o, w = dev[i % 2]
        session.search_device(o.data_ptr(), w.data_ptr(), q, K, d_s.data_ptr(), d_i.data_ptr(), stream.cuda_stream)

    check = StepCheck([d_s, d_i], lambda i: want[i % 2] if want is not None else None, args.steps)
    step_ms, kernel_ms, _ = timed_device(session, step, args.steps, args.warmup, flush, stream, world, check=check)
    host_ms, e2e_bad = [], 0
    res = (np.empty((q, K), np.float32), np.empty((q, K), np.int32))
    for i in range(args.warmup):
        session.search(sets[i % 2], K, out=res)
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        session.search(sets[i % 2], K, out=res)
        host_ms.append((time.perf_counter() - t0) * 1e3)
        if want is not None:
            e2e_bad += 0 if same_bits(res, want[i % 2]) else 1
    total = max_over_ranks(sum(step_ms), world)
    out.update({'value': world * q * args.steps / (total / 1e3), 'unit': UNIT, 'p50_ms': percentile(step_ms, 50),
                'p95_ms': percentile(step_ms, 95), 'main_kernel_ms_avg': sum(kernel_ms) / len(kernel_ms),
                'e2e': {'p50_ms': percentile(host_ms, 50), 'p95_ms': percentile(host_ms, 95),
                        'value': world * q * args.steps / (max_over_ranks(sum(host_ms), world) / 1e3)},
                'timed_parity': dict(check.report(), e2e_checked=len(host_ms) if want is not None else 0,
                                     e2e_mismatched=e2e_bad),
                'a5_median_over_e2e_p50': (sum(A5_PUBLISHED_MS.values()) / 2) / percentile(host_ms, 50)})
    session.close()
    return out


SERVE_RATES = (5000, 10000, 20000, 50000)  # --serve-all
SERVE_RATES_DEFAULT = (5000, 20000)
SERVE_TERMS, SERVE_KS, SERVE_POOL = (1, 16), (10, 100, 1000), 4096


def serve_leg(pkg, args, spec, index, local, rates=SERVE_RATES):
    """The serving loop on the 10M-doc index: open-loop Poisson arrivals at 5k-50k queries/s of
    1-16 terms (drawn by df) and K from {10, 100, 1000}; the continuous-batching server (learned
    pruning on, every result exact) against the plain engine serving one query per Search."""
    lo, hi = SERVE_TERMS
    qo, w = pkg.synthetic_queries(index.offsets, SERVE_POOL, lo, hi, 4242)
    ks = np.random.default_rng(4243).choice(SERVE_KS, SERVE_POOL).astype(np.int32)
    kmax = max(SERVE_KS)
    t = time.perf_counter()
    cap = 1024
    trainer = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=cap, word_capacity=cap * hi, max_k=kmax, device_id=local,
                                        prune=True)
    model = pkg.learned.fit(trainer, index.offsets, queries=args.mix_train_queries, ks=SERVE_KS, lo=lo, hi=hi,
                            seed=args.train_seed, steps=args.train_steps, batch=4096, gen_batch=cap,
                            target_fallback=args.target_fallback, device=f'cuda:{local}')
    trainer.close()
    log(f'serving model trained in {time.perf_counter() - t:.1f}s: {model.report}')
    session = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=256, word_capacity=256 * hi, max_k=kmax, device_id=local,
                                        prune=True)
    session.set_threshold_model(model)
    out = {'workload': WORKLOAD, 'arrivals': 'Poisson (open loop), seeded', 'terms': f'U{{{lo}..{hi}}} drawn by df',
           'k': 'per query from {10, 100, 1000}', 'query_pool': SERVE_POOL, 'runs': []}
    configs = (('plain, one query per Search', dict(max_batch=1, learned=False)),
               ('continuous batching, plain', dict(max_batch=256, learned=False, candidate_budget=64_000)),
               ('continuous batching, learned pruning', dict(max_batch=256, learned=True, candidate_budget=64_000)))
    for rate in rates:
        total = int(min(rate * args.serve_seconds, 40_000))
        for label, opts in configs:
            if opts['max_batch'] == 1 and rate > 10_000:
                continue  # saturated far below these rates: its queue only grows
            session.prepare_batch_graphs(opts['max_batch'], opts['learned'])  # as the server's creation does
            made = session.info()['graph_instantiations']
            lat, st = pkg.serving.serve_poisson(session, qo, w, ks, rate_qps=rate, total=total, seed=rate, **opts)
            made = session.info()['graph_instantiations'] - made
            row = {'config': label, 'offered_qps': rate, 'queries': total, 'achieved_qps': st['achieved_qps'],
                   'p50_ms': st['p50_us'] / 1e3, 'p95_ms': st['p95_us'] / 1e3, 'p99_ms': st['p99_us'] / 1e3,
                   'mean_batch': st['mean_batch'],
                   # graphs instantiated while serving (the server prepares every batch bucket's graph
                   # when it is created, before the first arrival)
                   'graphs_instantiated_while_serving': made}
            out['runs'].append(row)
            log(f'serve {row}')
    session.close()
    return out


def run_doc_sharded(args):
    """--shard docs: the 10M-doc index split by document range over the N ranks (one GPU each); every
    rank searches the same query batches over its range, the local top-K lists are all-gathered with
    NCCL (Q*K*8 bytes per rank) and merged on every rank by the merge kernel (ShardedSession).  A step
    is one Search of the batch; value = queries/s of the whole job (strong scaling: the corpus is fixed,
    each rank holds 1/N of it); steps timed with CUDA events on the launching stream, max over ranks."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank, world, local = setup_dist(args.gpus)
    torch.cuda.set_device(local)
    dist.init_process_group('nccl', timeout=timedelta(seconds=300), device_id=torch.device('cuda', local))
    pkg = importlib.import_module('bm25-npu_b200')
    from oracle import oracle
    spec, index = build_corpus(pkg, args.docs, args.vocab)
    data = oracle.contributions(index, spec.k1)  # the eager scores each rank slices its shard from
    sets = batches(pkg, index, 0)  # the same batches on every rank
    session = pkg.sharded.ShardedSession(index.offsets, index.docs, data, index.num_docs, query_capacity=Q,
                                         word_capacity=Q * TERMS, max_k=K)
    want = [oracle.search(index.offsets, index.docs, data, index.num_docs, *qs, K) for qs in sets] \
        if rank == 0 else None
    del data
    host_ok = []
    first_diff = None
    for i, qs in enumerate(sets):
        got = session.search(qs, K)
        if want is not None:
            host_ok.append(same_bits(got, want[i]))
            if not host_ok[-1] and first_diff is None:
                bad_q = [j for j in range(Q) if not same_bits((got[0][j], got[1][j]), (want[i][0][j], want[i][1][j]))]
                first_diff = {'batch': i, 'queries': bad_q, 'got': [got[0][bad_q[0]].tolist(), got[1][bad_q[0]].tolist()],
                              'want': [want[i][0][bad_q[0]].tolist(), want[i][1][bad_q[0]].tolist()]}
    parity = all(host_ok)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dev_sets = [(torch.from_numpy(o).cuda(), torch.from_numpy(w).cuda()) for o, w in sets]
    flush = torch.empty(64 << 20, dtype=torch.float32, device='cuda')
    for i in range(args.warmup):
        session.search_device(*dev_sets[i % 2], Q, K)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    checked = bad = 0
    dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.zero_()
        starts[i].record(stream)
        gs, gi = session.search_device(*dev_sets[i % 2], Q, K)
        ends[i].record(stream)
        if want is not None:  # outside the step's events
            checked += 1
            bad += 0 if same_bits((gs.cpu().numpy(), gi.cpu().numpy()), want[i % 2]) else 1
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total = max_over_ranks(sum(step_ms), world)
    dist.barrier()
    if rank == 0:
        print(json.dumps({
            'metric': METRIC, 'value': Q * args.steps / (total / 1e3), 'unit': UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total / args.steps,
            'higher_is_better': True, 'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': WORKLOAD, 'docs': spec.docs, 'queries': Q, 'terms': TERMS, 'k': K,
                       'parallelism': f'doc-sharded x{world} (NCCL all-gather of the local top-K, merge kernel)',
                       'l2': 'flushed between steps (256 MiB write)'},
            'parity': {'bit_exact': bool(parity and bad == 0), 'checked_searches': checked + len(sets),
                       'host_searches_exact': host_ok, 'timed_mismatched': bad, 'first_difference': first_diff,
                       'against': 'unsharded oracle'},
        }), flush=True)
    session.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def run_reference(args):
    rank, world, _ = setup_dist(args.gpus)
    if rank != 0:
        return 0
    pkg = importlib.import_module('bm25-npu_b200')
    spec, index = build_corpus(pkg)
    sets = batches(pkg, index, 0)
    res = cpu_search_leg(index, sets, K, budget_s=1e9, max_steps=args.steps, warmup=args.warmup)
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': res['value'], 'unit': UNIT, 'n_gpus': args.gpus,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': Q * 1e3 / res['value'],
        'p50_ms': res['p50_ms'], 'p95_ms': res['p95_ms'], 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': WORKLOAD, 'docs': spec.docs, 'vocab': spec.vocab, 'zipf_s': spec.zipf_s,
                   'len_mean': spec.len_mean, 'k1': spec.k1, 'b': spec.b, 'queries': Q, 'terms': TERMS, 'k': K},
        'cpu_baseline': {k2: res[k2] for k2 in ('value', 'unit', 'cores', 'kind', 'sample')},
        'e2e': {'value': res['value'], 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=60)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--shard', default='queries', choices=['queries', 'docs'],
                    help='queries: a replica per GPU (the default); docs: the index split by document range')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--tile-docs', type=int, default=0)
    ap.add_argument('--fan-in', type=int, default=0)
    ap.add_argument('--kernel', type=int, default=5,
                    help='0 streaming, 1 one CTA per (query, tile), 4 tile groups, 5 warp tiles')
    ap.add_argument('--stages', type=int, default=0)
    ap.add_argument('--chunk', type=int, default=0, help='postings per ring stage of the tile-group kernel')
    ap.add_argument('--docs', type=int, default=0, help='reduced corpus for profiling captures (not a bench line)')
    ap.add_argument('--vocab', type=int, default=0, help='reduced vocabulary for profiling captures')
    ap.add_argument('--no-learned', action='store_true', help='skip the learned-pruned leg')
    ap.add_argument('--train-queries', type=int, default=200_000)
    ap.add_argument('--train-steps', type=int, default=3000)
    ap.add_argument('--train-seed', type=int, default=7)
    ap.add_argument('--target-fallback', type=float, default=0.02)
    ap.add_argument('--no-mix', action='store_true', help='skip the batched 256-query mix')
    ap.add_argument('--mix-train-queries', type=int, default=120_000)
    ap.add_argument('--no-blockmax', action='store_true', help='skip the 4.2M-doc block-max workload')
    ap.add_argument('--no-refshape', action='store_true', help="skip the reference's own corpus shape at 10M docs")
    ap.add_argument('--blockmax-train-queries', type=int, default=200_000)
    ap.add_argument('--no-serve', action='store_true', help='skip the serving loop (Poisson arrivals)')
    ap.add_argument('--serve-all', action='store_true', help='serving loop at 5k, 10k, 20k and 50k queries/s')
    ap.add_argument('--serve-seconds', type=float, default=1.0)
    ap.add_argument('--no-tune', action='store_true', help='keep the default runtime tuning (no autotune)')
    args = ap.parse_args()
    if args.impl == 'reference':
        return run_reference(args)
    if args.shard == 'docs':
        if args.warmup < 3:
            args.warmup = 3
        return run_doc_sharded(args)
    if args.warmup < 3:
        args.warmup = 3

    import torch
    import torch.distributed as dist

    rank, world, local = setup_dist(args.gpus)
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=600), device_id=torch.device('cuda', local))
    pkg = importlib.import_module('bm25-npu_b200')
    spec, index = build_corpus(pkg, args.docs, args.vocab)
    df = index.df()
    sets = batches(pkg, index, rank)
    t = time.perf_counter()
    session = pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                        query_capacity=Q, word_capacity=Q * TERMS, max_k=K, device_id=local,
                                        tile_docs=args.tile_docs, merge_fan_in=args.fan_in, kernel=args.kernel,
                                        ring_stages=args.stages, ring_chunk=args.chunk,
                                        prune=args.kernel in (4, 5) and not args.no_learned)
    info = session.info()
    log(f'engine ready in {time.perf_counter() - t:.1f}s: {info}')
    tuning = None
    if info['kernel'] == 5 and not args.no_tune:
        # runtime knobs timed on a sample batch of the same shape (not one of the timed batches);
        # every combination is bit-checked against the first, and the fastest is kept
        t = time.perf_counter()
        sample = pkg.synthetic_queries(index.offsets, Q, TERMS, TERMS, SEED_A + 77 + 1000 * rank)
        best, table = pkg.autotune.tune(session, sample, K, space={'claim_tiles': (2, 4, 8),
                                                                   'tail_claims': (1, 2, 4)}, reps=8)
        tuning = {'chosen': {key: best[key] for key in ('claim_tiles', 'tail_claims')},
                  'sample': f'one batch of {Q} x {TERMS} words (its own seed), 8 timed Searches per setting',
                  'ms': {f"{c['claim_tiles']}x{c['tail_claims']}": round(ms, 4) for c, ms in table},
                  'seconds': round(time.perf_counter() - t, 2)}
        log(f'tuning: {tuning}')

    # Parity of both batches against the CPU oracle (outside every timer).
    parity = None
    want = None
    if rank == 0:
        from oracle import oracle
        data = oracle.contributions(index, spec.k1)
        ok = True
        want = []
        for qs in sets:
            rs, ri = oracle.search(index.offsets, index.docs, data, index.num_docs, *qs, K)
            want.append((rs, ri))
            gs, gi = session.search(qs, K)
            ok &= bool(np.array_equal(gi, ri) and np.array_equal(gs.view(np.uint32), rs.view(np.uint32)))
        parity = {'batches': len(sets), 'bit_exact': ok, 'against': 'oracle (C restatement, eager FP32)'}
        del data
        log(f'parity vs oracle: {parity}')

    stream = torch.cuda.Stream()
    dev_sets = [(torch.from_numpy(o).cuda(), torch.from_numpy(w).cuda()) for o, w in sets]
    d_scores = torch.empty((Q, K), dtype=torch.float32, device='cuda')
    d_ids = torch.empty((Q, K), dtype=torch.int32, device='cuda')
    flush = torch.empty(64 << 20, dtype=torch.float32, device='cuda')  # 256 MiB > 126 MB L2
    bytes_per = [algorithmic_bytes(df, index.vocab, o, w, K) for o, w in sets]
    distinct_per = [algorithmic_bytes(df, index.vocab, o, w, K, distinct=True) for o, w in sets]

    def device_step(i):
        o, w = dev_sets[i % 2]
        session.search_device(o.data_ptr(), w.data_ptr(), Q, K, d_scores.data_ptr(), d_ids.data_ptr(),
                              stream.cuda_stream)

    check = StepCheck([d_scores, d_ids], lambda i: want[i % 2] if want is not None else None, args.steps)
    step_ms, kernel_ms, clock_info = timed_device(session, device_step, args.steps, args.warmup, flush, stream,
                                                  world, Clocks(local), check=check)
    plain_stats = session.search_stats(reset=True)
    total_ms = max_over_ranks(sum(step_ms), world)
    value = world * Q * args.steps / (total_ms / 1e3)

    # End to end through the C ABI with host buffers (pinned arenas, H2D/D2H inside the call).
    host_ms = []
    out = (np.empty((Q, K), np.float32), np.empty((Q, K), np.int32))
    for i in range(args.warmup):
        session.search(sets[i % 2], K, out=out)
    if world > 1:
        dist.barrier()
    e2e_checked = e2e_bad = 0
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        session.search(sets[i % 2], K, out=out)
        host_ms.append((time.perf_counter() - t0) * 1e3)
        if want is not None:  # outside the timer: every e2e result against the oracle
            e2e_checked += 1
            e2e_bad += 0 if same_bits(out, want[i % 2]) else 1
    if parity is not None:
        parity['timed'] = dict(check.report(), e2e_checked=e2e_checked, e2e_mismatched=e2e_bad)
        parity['bit_exact'] = bool(parity['bit_exact'] and check.mismatched == 0 and e2e_bad == 0)
    e2e_total = sum(host_ms)
    if world > 1:
        tt = torch.tensor([e2e_total], device='cuda', dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_total = float(tt.item())
    e2e_value = world * Q * args.steps / (e2e_total / 1e3)
    word_offset = -(-((Q + 1) * 8) // 32) * 32
    h2d = -(-(word_offset + Q * TERMS * 4) // 32) * 32
    id_off = -(-(Q * K * 4) // 32) * 32
    d2h = -(-(id_off + Q * K * 4) // 32) * 32 + 32

    # Roofline of the dominant kernel: algorithmic bytes / its event-timed duration, launch by launch
    # (events recorded by the engine on the launching stream around that one kernel).
    bytes_total = sum(bytes_per[i % 2] for i in range(args.steps))
    bytes_avg = bytes_total / args.steps
    achieved = bytes_total / (sum(kernel_ms) / 1e3) / 1e9
    search_achieved = bytes_total / (sum(step_ms) / 1e3) / 1e9
    launches_per_search = 1 if info['kernel'] == 1 else 3
    peak, peak_kind = hbm_peak()
    traffic = traffic_from_profile({0: 'stream_search_kernel_synthetic_10m.txt',
                                    4: 'tile_group_kernel_synthetic_10m.txt',
                                    5: 'warp_tile_kernel_synthetic_10m.txt'}.get(info['kernel'], '-'))
    if args.docs or args.vocab:
        traffic = None  # the profiles cover the full-size workload

    learned = None
    if info['kernel'] in (4, 5) and not args.no_learned:
        learned = learned_leg(pkg, args, spec, index, session, sets, want, flush, stream, dev_sets, local, world)
        learned['speedup_vs_plain'] = learned['learned']['value'] / value
        learned['e2e_speedup_vs_plain'] = learned['learned']['e2e']['value'] / e2e_value
        learned['plain_per_search'] = {key: v / args.steps for key, v in plain_stats.items()}

    serving = None
    if info['kernel'] in (4, 5) and not args.no_serve and world == 1 and not (args.docs or args.vocab):
        serving = serve_leg(pkg, args, spec, index, local, SERVE_RATES if args.serve_all else SERVE_RATES_DEFAULT)

    mix = blockmax = refshape = None
    full_size = info['kernel'] in (4, 5) and not (args.docs or args.vocab)
    session_open = True
    if full_size and not (args.no_mix and args.no_blockmax and args.no_refshape):
        session.close()  # frees the 10M index before the next corpus is resident
        session_open = False
    if full_size and not args.no_refshape:
        refshape = refshape_leg(pkg, args, local, world, flush, stream, rank)
    if full_size and not args.no_mix:
        mix = mix_leg(pkg, args, local, world, flush, stream, rank)
    if full_size and not args.no_blockmax:
        blockmax = blockmax_leg(pkg, args, local, world, flush, stream, rank)

    cpu = cpu_bm25s = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res = cpu_search_leg(index, sets, K, budget_s=20.0, max_steps=40)
        cpu = {k2: res[k2] for k2 in ('value', 'unit', 'cores', 'kind', 'sample')}
        cpu_bm25s = cpu_bm25s_leg(index, spec.k1, sets, want)

    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
            'p50_ms': percentile(step_ms, 50), 'p95_ms': percentile(step_ms, 95),
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': WORKLOAD if not (args.docs or args.vocab) else f'{WORKLOAD}_reduced', 'docs': spec.docs, 'vocab': spec.vocab, 'zipf_s': spec.zipf_s,
                       'len_mean': spec.len_mean, 'len_sigma': spec.len_sigma, 'k1': spec.k1, 'b': spec.b,
                       'postings': index.postings, 'queries': Q, 'terms': TERMS, 'k': K,
                       'batches': 'A/B alternating, terms drawn by df', 'l2': 'flushed between steps (256 MiB write)',
                       'tile_docs': info['tile_docs'], 'tiles': info['tiles'], 'merge_fan_in': info['merge_fan_in'],
                       'merge_levels': info['merge_levels'], 'kernel': info['kernel'],
                       'ring_stages': info['ring_stages'], 'ring_chunk': info['ring_chunk'], 'grid': info['grid'],
                       'parallelism': f'replicas x{world} (queries sharded)'},
            'e2e': {'value': e2e_value, 'unit': UNIT, 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                    'p50_ms': percentile(host_ms, 50), 'p95_ms': percentile(host_ms, 95),
                    'path': 'bm25_search (C ABI, host buffers): pack + CUDA graph (H2D, kernel, D2H) + validate'},
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'traffic': traffic, 'peak_source': peak_kind,
                         'algorithmic_bytes_per_launch': bytes_avg,
                         'distinct_word_bytes_per_launch': sum(distinct_per[i % 2] for i in range(args.steps)) / args.steps,
                         'kernel_ms_avg': sum(kernel_ms) / len(kernel_ms),
                         'kernel_share_of_step': sum(kernel_ms) / sum(step_ms),
                         'search_achieved_gbs': search_achieved,
                         'kernel': {0: 'bm25k::StreamSearchKernel', 1: 'bm25k::TileSearchKernel',
                                    4: 'bm25k::TileGroupKernel', 5: 'bm25k::WarpTileKernel'}[info['kernel']]},
            'gpu_launches': args.steps * launches_per_search,
            'clocks': clock_info,
            'parity': parity,
        }
        if tuning is not None:
            line['tuning'] = tuning
        if learned is not None:
            line['learned_pruned'] = learned
        if mix is not None:
            line['batched_mix'] = mix
        if blockmax is not None:
            line['blockmax_c4'] = blockmax
        if refshape is not None:
            line['reference_shape'] = refshape
        if serving is not None:
            line['serving'] = serving
        if cpu is not None:
            line['cpu_baseline'] = cpu
        if cpu_bm25s is not None:
            line['cpu_baseline_bm25s'] = cpu_bm25s
        print(json.dumps(line), flush=True)
    if session_open:
        session.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == '__main__':
    sys.exit(main())
