#!/usr/bin/env python3
"""Throughput of the MLEbfgs localization path (GS2D 7x7 single-emitter fits/s).

One step = one localization call over N = 100,000 synthetic 7x7 ROI records
(the reference's per-call batch size, MaxPointNum = 102,400): WLE pre-pass
(PSF width, nearest neighbour, molecule type) -> single-emitter fit with the
reference's fixed schedule -> CRLB, all on the device through the C ABI
(qcs_loc_localize_device).  Records: seeded synthetic 7x7 ROIs (sigma
U(1.0,1.6) px, photons log-U[500,5000], background U(20,100) e-/px, Poisson),
16 distinct batches rotated across steps (179 MB of records, more than the
126 MB L2).  The `frames` object adds the whole-frame pipeline (2048 x 2048
frames -> extraction -> multi-emitter localization -> CRLB) in frames/s.

Printed JSON line (rank 0): `value` is device-timed fits/s with records
resident in HBM, three localization contexts used in turn on three streams
(one call's latency-bound tail overlaps the next calls' kernels;
`value_one_stream` is one context on one stream); `e2e` is the same metric
through the asynchronous host-buffer calls (qcs_loc_localize_async +
qcs_loc_finish on three contexts in turn, so one call stays queued while the
host reads another's rows: pinned host records in, rows and counters out, every copy
inside the timed region; `e2e.sync_value`: the synchronous
qcs_loc_bfgs_mle_localization, one call at a time); `roofline` is the fit kernel against the measured
special-function-unit rate (the loss is exp/log bound, not HBM or tensor
bound); `cpu_baseline` is the reference's own code compiled for the host
(oracle/_ref) on all host cores.

--impl reference times the reference's CPU implementation of the same step
(oracle/_ref/libqcs_ref_host.so: the reference sources compiled for the CPU,
WLE + localization + CRLB) on all host cores, rank 0 only.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "qc-storm_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

METRIC = "7x7 fits/s on 1 B200: learned-init vs plain MLEbfgs at equal RMSE/CRLB"
UNIT = "fits/s"
N_PER_STEP = 100_000
BATCHES = 16
R = 7
PX_EVALS_PER_FIT = 176 * R * R  # reference schedule: 176 loss evaluations of R*R pixels
MUFU_PER_PX_EVAL = 2            # exp of the model, log of the model (log of the data is invariant)
# DRAM bytes (read + write) per fit of fit_single_kernel<7, GS2D>, from one ncu capture of
# `bench.py --profile-fit 200000` (profiles/fit_single_gs2d7_200k_full.md: 27.28 MB read, 0 B
# written for 200 k fits: the rows stay in L2 during the launch); algorithmic: 112 B record +
# 24 B WLE row read, 48 B row written.
DRAM_BYTES_PER_FIT = (27.277056e6 + 0.0) / 2e5
ALGO_BYTES_PER_FIT = 112 + 24 + 48


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def start_clock_sampler(gpu_index):
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + q, "--format=csv,noheader,nounits", "-i", str(gpu_index),
                              "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL)
    except OSError:
        p = None
    return p, f.name


def stop_clock_sampler(p, path, t_start, t_end):
    """Median SM clock and active throttle reasons of the samples taken
    between host times t_start and t_end."""
    import datetime
    out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    if p is None:
        return out
    p.terminate()
    try:
        p.wait(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    with open(path) as fh:
        for line in fh:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                if ts < t_start or ts > t_end:
                    continue
                sm.append(float(parts[2]))
                mx.append(float(parts[3]))
            except ValueError:
                continue
            for name, v in zip(names, parts[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(name)
    os.unlink(path)
    if sm:
        out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
               "samples": len(sm)}
    return out


def batch_seed(rank, b):
    """Seed of record batch b on `rank`: every rank localizes records of its own
    (weak scaling; the path has no data-path collective)."""
    return 1000 * rank + b


def max_over_ranks(ms, dist):
    """The slowest rank's time (ms) when several ranks run: all-reduce MAX, on
    the GPU under NCCL, on the CPU under gloo."""
    if dist is None:
        return ms
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def device_timed(steps, warmup, enqueue, streams, dist):
    """Device time (ms, the slowest rank's) of `steps` calls enqueue(k, stream)
    after `warmup` untimed ones.  With several streams the calls rotate over
    them (as many contexts in turn), so one call's latency-bound tail overlaps
    the next calls' kernels; the CUDA events bracket every stream."""
    import torch
    for k in range(warmup):
        enqueue(k, streams[k % len(streams)])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    a = streams[0]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(a)
    for s in streams[1:]:
        s.wait_event(e0)
    for k in range(steps):
        enqueue(k, streams[k % len(streams)])
    for s in streams[1:]:
        ev = torch.cuda.Event()
        ev.record(s)
        a.wait_event(ev)
    e1.record(a)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    return max_over_ranks(e0.elapsed_time(e1), dist)


MIN_TIMED_MS = 1000.0  # the K-step window is repeated until the device-timed total reaches this


def device_timed_windows(steps, warmup, enqueue, streams, dist):
    """device_timed over windows of exactly `steps` calls, repeated until the
    windows add up to MIN_TIMED_MS of device time (so the clock sampler, which
    polls every 200 ms, sees the timed region); returns (median window ms,
    window count).  The count follows from the first window's slowest-rank
    time, so every rank runs the same windows."""
    first = device_timed(steps, warmup, enqueue, streams, dist)
    more = 0 if first >= MIN_TIMED_MS else min(int(math.ceil(MIN_TIMED_MS / max(first, 1e-3))) - 1, 500)
    windows = [first] + [device_timed(steps, 0, enqueue, streams, dist) for _ in range(more)]
    return statistics.median(windows), len(windows)


def job_rate(steps, per_step, world, ms):
    """Whole-job rate: every rank's records over the slowest rank's time."""
    return steps * per_step * world / (ms * 1e-3)


def cpu_reference_rate(steps=1, per_thread=6000, threads=None):
    """fits/s of the reference's own code compiled for the host (oracle/_ref),
    WLE + localization + CRLB, one chunk of records per host thread; falls back
    to the CPU oracle restatement when the reference build is absent."""
    import oracle_lib as O
    from qcstorm_b200 import synth
    threads = threads or os.cpu_count() or 1
    ref = O.ref_host()
    kind = "reference" if ref is not None else "port"
    lib = "ref" if ref is not None else "oracle"
    if lib == "oracle":
        O.set_threads(1)
    chunks = []
    for t in range(threads):
        rec, para, _ = synth.gs2d_rois(per_thread, R=R, seed=9000 + t)
        chunks.append((rec, para))
    rates = []
    for _ in range(steps):
        done = [0] * threads

        def work(i):
            rec, para = chunks[i]
            w = O.wle(para, rec, lib)
            O.localize(para, rec, w, lib)
            done[i] = rec.shape[0]

        t0 = time.perf_counter()
        ths = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        dt = time.perf_counter() - t0
        rates.append(sum(done) / dt)
    return {"value": max(rates) if steps == 1 else statistics.median(rates), "unit": UNIT, "cores": threads,
            "kind": kind,
            "sample": "%d GS2D 7x7 records per host thread x %d threads per step (WLE + fit + CRLB)" % (
                per_thread, threads)}, rates


# loss evaluations of the reference's fixed schedules (2P initial gradient, IT iterations of 12 line-search
# evaluations, IT - 1 more gradients) and MUFU operations per pixel-evaluation (exps of the model + its log)
SCHEDULE_EVALS = {"gs2d": 176, "as3d": 264, "2e": 364, "3e": 544}
MUFU_PER_EVAL = {"gs2d": 2, "as3d": 2, "2e": 3, "3e": 4}


def cascade_mufu_ops(R, single, n2=0, n3=0, single_kind="gs2d"):
    """MUFU operations the fits of one localization call execute on the
    reference schedule: queue lengths of the single-emitter, 2E and 3E stages."""
    px = R * R
    return px * (single * SCHEDULE_EVALS[single_kind] * MUFU_PER_EVAL[single_kind] +
                 n2 * SCHEDULE_EVALS["2e"] * MUFU_PER_EVAL["2e"] + n3 * SCHEDULE_EVALS["3e"] * MUFU_PER_EVAL["3e"])


def threaded_cpu_rate(make_sample, work, threads=None):
    """Units per second of work(sample) run on one prepared sample per host
    thread (ctypes releases the GIL, so the threads run in parallel)."""
    threads = threads or os.cpu_count() or 1
    samples = [make_sample(t) for t in range(threads)]
    done = [0] * threads

    def run(i):
        done[i] = work(samples[i])

    t0 = time.perf_counter()
    ths = [threading.Thread(target=run, args=(i,)) for i in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return sum(done) / (time.perf_counter() - t0), threads


def shape_cpu_baseline(kind, R, per_thread):
    """The reference's code compiled for the host (oracle/_ref) on every host
    core over a bounded sample of the workload: WLE + fit (+ cascade) + CRLB.
    AS3D 9x9 runs the reference's 9x9 kernel directly (its own dispatcher
    would run the 8x8 one)."""
    import oracle_lib as O
    from qcstorm_b200 import synth
    if O.ref_host() is None:
        return None
    gen = synth.as3d_rois if kind == "as3d" else synth.multi_rois

    def make(t):
        rec, para, _ = gen(per_thread, R=R, seed=9500 + t)
        return rec, para

    def work(sample):
        rec, para = sample
        w = O.wle(para, rec, "ref")
        if kind == "as3d":
            O.crlb(para, O.fit_single(1, para, rec, w, lib="ref"), lib="ref")
        else:
            O.localize(para, rec, w, lib="ref")
        return rec.shape[0]

    rate, threads = threaded_cpu_rate(make, work)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": "%d %s %dx%d records per host thread x %d threads (WLE + fit%s + CRLB)" % (
                per_thread, kind, R, R, threads, "" if kind == "as3d" else " cascade")}


def frame_cpu_baseline(frames_per_thread=1):
    """frames/s of the frame pipeline on every host core, one frame per
    thread: ROI extraction by the oracle port (bit-pinned to the reference's
    host build, which runs its CUDA extraction kernels through a SIMT emulator
    at ~26 s per 2048 x 2048 frame and would misstate a CPU's speed), then the
    reference's host build for WLE + localization cascade + CRLB."""
    import oracle_lib as O
    from qcstorm_b200 import synth
    if O.ref_host() is None:
        return None
    O.set_threads(1)

    def make(t):
        fr, para, _ = synth.frames(frames_per_thread, width=FRAME_W, height=FRAME_H, density=3000, seed=9700 + t)
        para.MultiEmitterFitEn = 1
        return fr, para

    def work(sample):
        fr, para = sample
        rois, _, _, _ = O.extract(para, fr, 1, lib="oracle")
        O.localize(para, rois, O.wle(para, rois, "ref"), lib="ref")
        return fr.shape[0]

    rate, threads = threaded_cpu_rate(make, work)
    O.set_threads(0)
    return {"value": rate, "unit": "frames/s", "cores": threads, "kind": "port+reference",
            "sample": "%d 2048x2048 frame(s) per host thread x %d threads: extraction by the oracle port, WLE + "
                      "localization cascade + CRLB by the reference's host build" % (frames_per_thread, threads)}


def run_reference_arm(args, rank):
    if rank != 0:
        return 0
    base, rates = cpu_reference_rate(steps=args.warmup + args.steps)
    rates = rates[args.warmup:]
    v = statistics.median(rates)
    base["value"] = v
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": env_int("WORLD_SIZE", 1),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * N_PER_STEP / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_dict(args),
        "cpu_baseline": base,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_dict(args):
    return {
        "workload": "GS2D 7x7 single-emitter MLEbfgs, %d ROI records per call: WLE pre-pass + fit + CRLB; "
                    "sigma U(1.0,1.6) px, photons log-U[500,5000], background U(20,100) e-/px" % N_PER_STEP,
        "roi_size": R, "rois_per_step": N_PER_STEP, "mode": "plain MLEbfgs, reference schedule, bit-exact with "
                                                          "the reference CUDA kernel",
        "input_batches": BATCHES, "l2": "records rotate over %d batches (%.0f MB > 126 MB L2)" % (
            BATCHES, BATCHES * N_PER_STEP * R * (R + 1) * 2 / 1e6),
        "parallelism": "dp%d (independent frame batches per GPU)" % args.gpus,
    }


FRAME_W = FRAME_H = 2048
FRAMES = 8             # distinct frames rotated across steps (2048 x 2048 uint16 = 8.4 MB each)
FRAMES_PER_CALL = 32   # frames whose ROIs accumulate before one localization call
MAX_POINT_NUM = 102400


TRAIN_FRAMES = 32      # frames (seeds disjoint from the timed ones) whose records train the frame network
COUNT_TH = 0.5         # emitter-count routing threshold of the learned frame pipeline


def frame_truth_match(rows, truth, radius=1.0):
    """Distance (px) of each localization to the nearest true emitter of its
    frame (frame f holds the emitters of distinct frame f % FRAMES); rows with
    no emitter within `radius` count as unmatched."""
    from scipy.spatial import cKDTree
    rows = rows[rows[:, 0] > 0]
    frame = rows[:, 11].astype(np.int64)
    dist = np.full(rows.shape[0], np.inf)
    for f in np.unique(frame):
        t = truth[int(f) % len(truth)]
        sel = frame == f
        d, _ = cKDTree(np.stack([t["x"], t["y"]], 1)).query(np.stack([rows[sel, 1], rows[sel, 2]], 1))
        dist[sel] = d
    ok = dist < radius
    return {"localizations": int(rows.shape[0]), "matched": int(ok.sum()),
            "rmse_px": float(np.sqrt(np.mean(dist[ok] ** 2))) if ok.any() else None}


def train_frame_net(para, stream, seed=9001, multi_starts=False):
    """The network of the learned frame pipeline, trained on the GPU on the
    records that extraction cuts from TRAIN_FRAMES fresh frames (same
    generator, other seeds): start-point targets from the records the plain
    multi-emitter cascade kept single, emitter-count classes from its outcome
    (qcs_loc_count_labels_device).  With multi_starts, also two- and
    three-emitter start-point networks on the same records, attached.
    Returns (net, info, extra networks)."""
    import torch
    from qcstorm_b200 import lib, synth
    sh = stream.cuda_stream
    t0 = time.perf_counter()
    fr, _, _ = synth.frames(TRAIN_FRAMES, width=FRAME_W, height=FRAME_H, density=3000, seed=seed)
    ex = lib.ExtractContext(para, max_batched_num=1, capacity=MAX_POINT_NUM)
    loc = lib.LocContext(para, capacity=MAX_POINT_NUM)
    d_fr = torch.from_numpy(fr.view(np.int16)).cuda()
    fb = FRAME_W * FRAME_H * 2
    torch.cuda.synchronize()
    for f in range(TRAIN_FRAMES):
        ex.extract_device(d_fr.data_ptr() + f * fb, 1, f, stream=sh)
    n = ex.accumulated()
    d_rois, d_wle, _ = ex.device_records()
    if multi_starts:
        lib.set_three_emitter_capture(loc)
    loc.localize_device(d_rois, n, d_wle, sh)
    labels = lib.count_labels(loc, n, sh)
    feat, scale = lib.LearnedNet.features(para, d_rois, n, stream=sh)
    tgt, valid = lib.LearnedNet.targets(para, d_rois, loc.device_rows(), scale, n, stream=sh)
    stream.synchronize()
    valid = valid * (labels == 0).float()
    counts = [int(c) for c in torch.bincount(labels.long(), minlength=3).cpu()]
    torch.cuda.synchronize()
    net = lib.LearnedNet(batch=4096, seed=5)
    losses = net.train(feat, tgt, valid, epochs=TRAIN_EPOCHS, lr=2e-3, stream=sh, classes=labels)
    stream.synchronize()
    extra = []
    if multi_starts:
        dr = _DevPtr(d_rois)
        net2 = train_two_emitter_net(loc, para, dr, feat, scale, n, R, TRAIN_EPOCHS, stream)
        net3 = train_three_emitter_net(loc, para, dr, feat, scale, n, R, TRAIN_EPOCHS, stream)
        net.set_two_emitter(net2, iters=TWO_ITERS, bisections=6, fallback="none")
        net.set_three_emitter(net3, iters=THREE_ITERS, bisections=6, dev_th=-1.0)
        net.set_direct_two_emitter(True)
        extra = [net2, net3]
    info = {"frames": TRAIN_FRAMES, "records": n, "epochs": TRAIN_EPOCHS, "seconds": time.perf_counter() - t0,
            "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
            "class_counts": counts,
            "labels": "plain multi-emitter cascade on this GPU: fits of the records it kept single, and its "
                      "outcome per record (0: kept single, 1: kept by the 2E fit, 2: passed on to the 3E fit)"}
    ex.close()
    loc.close()
    return net, info, extra


class _DevPtr:
    """A raw device address where a helper expects a tensor's data_ptr()."""

    def __init__(self, ptr):
        self.ptr = ptr

    def data_ptr(self):
        return self.ptr


def frame_pipeline(stream, steps, warmup, e2e=True, dist=None, world=1, net=None):
    """Whole-frame pipeline: 2048 x 2048 uint16 frames -> ROI extraction
    (background, smoothing, detection, 7x7 cut, WLE; one frame per extraction
    batch, records accumulating on the device) -> after FRAMES_PER_CALL frames
    one multi-emitter MLEbfgs call (1E -> 2E -> 3E cascade) -> CRLB, as the
    reference's plug-ins accumulate ROIs across extraction batches before
    localizing.  Everything runs on one stream with no host synchronisation
    (the record count stays on the device).  value: frames/s with frames
    resident in HBM; e2e: the same with every frame copied from pinned host
    memory and the rows read back to the host (qcs_loc_read_rows) inside the
    timed region.  With net, the localization call is the learned one
    (qcs_learned_localize_device_n: start points and emitter-count classes
    from the network, LEARNED_ITERS x LEARNED_BISECTIONS single-emitter fits,
    plain refits, the 2E / 3E stages); `accuracy` compares the first call's
    localizations with the generator's emitters."""
    import torch
    from qcstorm_b200 import lib, synth
    fr, para, truth = synth.frames(FRAMES, width=FRAME_W, height=FRAME_H, density=3000, seed=77)
    para.MultiEmitterFitEn = 1
    ex = lib.ExtractContext(para, max_batched_num=1, capacity=MAX_POINT_NUM)
    loc = lib.LocContext(para, capacity=MAX_POINT_NUM)
    d_fr = torch.from_numpy(fr.view(np.int16)).cuda()
    h_fr = torch.from_numpy(fr.view(np.int16)).pin_memory()
    sh = stream.cuda_stream
    frame_bytes = FRAME_W * FRAME_H * 2

    def call(k, e, l, s, host):
        """Call k on extraction context e, localization context l, stream handle s."""
        rois, wle, n = e.device_records()
        e.reset(s)
        for j in range(FRAMES_PER_CALL):
            f = k * FRAMES_PER_CALL + j
            if host:
                e.extract_device(h_fr.data_ptr() + (f % FRAMES) * frame_bytes, 1, f, stream=s, source="pinned")
            else:
                e.extract_device(d_fr.data_ptr() + (f % FRAMES) * frame_bytes, 1, f, stream=s)
        if net is None:
            l.localize_device_n(rois, wle, n, MAX_POINT_NUM, s)
        else:
            net.localize_n(l, rois, wle, n, MAX_POINT_NUM, iters=LEARNED_ITERS, bisections=LEARNED_BISECTIONS, stream=s)

    def step(k, host=False):
        call(k, ex, loc, sh, host)

    step(0)
    rows0, ratios0 = loc.read_rows(sh)
    recs0 = ex.accumulated()
    assert ex.dropped() == 0
    accuracy = frame_truth_match(rows0, truth)
    for k in range(warmup):
        step(k)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        step(k)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist) / steps
    # the same call sequence captured once in a CUDA graph and replayed
    # (every frame pointer repeats each call: 32 frames per call over 8 distinct)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
        step(0)
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            g.replay()
    torch.cuda.synchronize()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(steps):
            g.replay()
    g1.record(stream)
    torch.cuda.synchronize()
    ms_graph = max_over_ranks(g0.elapsed_time(g1), dist) / steps
    rows_g, _ = loc.read_rows(sh)
    assert rows_g.shape == rows0.shape
    del g
    # end to end: IN_FLIGHT (extraction, localization) context pairs on their own streams, so that the next calls'
    # frame copies and extractions run while a call localizes and its rows are read
    e2e_steps = max(6, steps // 4) if e2e else 1
    more = [(lib.ExtractContext(para, max_batched_num=1, capacity=MAX_POINT_NUM),
             lib.LocContext(para, capacity=MAX_POINT_NUM), torch.cuda.Stream()) for _ in range(IN_FLIGHT - 1)]
    pairs = [(ex, loc, sh)] + [(e, l, st.cuda_stream) for e, l, st in more]
    depth = len(pairs)
    for k in range(depth):
        call(k, *pairs[k], True)
        pairs[k][1].read_rows(pairs[k][2])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out_rows = 0
    for k in range(e2e_steps):
        if k >= depth:
            _, l, s = pairs[k % depth]
            out_rows += l.read_rows(s)[0].shape[0]
        call(k, *pairs[k % depth], True)
    for k in range(max(0, e2e_steps - depth), e2e_steps):
        _, l, s = pairs[k % depth]
        out_rows += l.read_rows(s)[0].shape[0]
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, dist) / e2e_steps
    for e, l, _ in pairs:
        e.close()
        l.close()
    call_name = "qcs_loc_localize_device_n" if net is None else "qcs_learned_localize_device_n"
    return {
        "workload": "2048x2048 uint16 frames, ~3000 emitters/frame (20%% in pairs < 3 px), GS2D 7x7, multi-emitter "
                    "fitting on; %d frames per localization call, %d distinct frames rotated" % (
                        FRAMES_PER_CALL, FRAMES),
        "frames_per_s": world * FRAMES_PER_CALL * 1e3 / ms, "ms_per_call": ms, "frames_per_call": FRAMES_PER_CALL,
        "records_per_call": recs0, "rows_per_call": int(rows0.shape[0]),
        "single_emitter_fits_per_call": int(round(float(ratios0[0]) * recs0)),
        "stages": {"single": int(round(float(ratios0[0]) * recs0)), "two_emitter": int(round(float(ratios0[1]) * recs0)),
                   "three_emitter": int(round(float(ratios0[2]) * recs0))},
        "graph": {"frames_per_s": world * FRAMES_PER_CALL * 1e3 / ms_graph, "ms_per_call": ms_graph,
                  "note": "one call (reset, %d extractions, localization) captured in a CUDA graph and replayed"
                          % FRAMES_PER_CALL},
        "localizations_per_s": world * rows0.shape[0] * 1e3 / ms, "steps": steps,
        "accuracy": dict(accuracy, basis="first call's localizations against the generator's emitters of their "
                                         "frames (nearest within 1 px)"),
        "e2e": {"frames_per_s": world * FRAMES_PER_CALL * 1e3 / e2e_ms, "ms_per_call": e2e_ms,
                "h2d_bytes_per_call": FRAMES_PER_CALL * frame_bytes,
                "d2h_bytes_per_call": int(out_rows / e2e_steps) * 48 + 32,
                "calls": "%d x qcs_extract_molecules (pinned frame) -> %s -> qcs_loc_read_rows, %d context pairs "
                         "on their streams in turn" % (FRAMES_PER_CALL, call_name, IN_FLIGHT)},
    }


def frame_pipeline_learned(stream, steps, warmup, dist=None, world=1, multi_starts=False):
    """The frame pipeline with the learned localization call, after training
    its network on records of other frames; with multi_starts, also two- and
    three-emitter start points, poor bright single fits routed straight to
    the two-emitter fit and no plain refits of the multi-emitter stages."""
    from qcstorm_b200.abi import default_para
    # the camera of synth.frames, multi-emitter fitting on (as in frame_pipeline)
    para = default_para(Offset=100.0, KAdc=0.45, QE=1.0, ImageWidth=FRAME_W, ImageHigh=FRAME_H, MultiEmitterFitEn=1)
    net, info, extra = train_frame_net(para, stream, multi_starts=multi_starts)
    net.set_count_threshold(COUNT_TH)
    r = frame_pipeline(stream, steps, warmup, e2e=True, dist=dist, world=world, net=net)
    net.fused_status()
    net.close()
    for x in extra:
        x.close()
    r["train"] = info
    r["count_threshold"] = COUNT_TH
    r["schedule"] = "%d BFGS iterations x %d line-search steps from the network's start points" % (
        LEARNED_ITERS, LEARNED_BISECTIONS)
    return r


LEARNED_ITERS = 2          # BFGS iterations from the network's start points (plain: 8)
LEARNED_BISECTIONS = 6     # line-search steps per iteration (plain: 11)
TRAIN_RECORDS = 200_000    # training records, same generator, seeds disjoint from the timed batches
TRAIN_EPOCHS = 8


def train_learned_net(para, stream, seed=4242, arch="mlp", lr=2e-3):
    """Train the start-point network (arch "mlp" or "conv") on the GPU:
    TRAIN_RECORDS fresh records labelled by plain fits, features and targets
    on the device, Adam over TRAIN_EPOCHS epochs (qcs_learned_train_device).
    Returns (net, info)."""
    import torch
    from qcstorm_b200 import lib, synth
    sh = stream.cuda_stream
    t0 = time.perf_counter()
    tr, _, _ = synth.gs2d_rois(TRAIN_RECORDS, R=R, seed=seed)
    d_tr = torch.from_numpy(tr.view(np.int16)).cuda()
    ctx = lib.LocContext(para, capacity=TRAIN_RECORDS)
    ctx.localize_device(d_tr.data_ptr(), TRAIN_RECORDS, 0, sh)
    stream.synchronize()
    feat, scale = lib.LearnedNet.features(para, d_tr.data_ptr(), TRAIN_RECORDS, stream=sh)
    tgt, valid = lib.LearnedNet.targets(para, d_tr.data_ptr(), ctx.device_rows(), scale, TRAIN_RECORDS, stream=sh)
    net = lib.LearnedNet(batch=4096, seed=5, arch=arch)
    stream.synchronize()
    t1 = time.perf_counter()
    losses = net.train(feat, tgt, valid, epochs=TRAIN_EPOCHS, lr=lr, stream=sh)
    stream.synchronize()
    info = {"records": TRAIN_RECORDS, "epochs": TRAIN_EPOCHS, "seconds": time.perf_counter() - t0,
            "training_seconds": time.perf_counter() - t1, "lr": lr,
            "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
            "labels": "plain MLEbfgs fits of the training records on this GPU"}
    ctx.close()
    return net, info


E2E_STEPS = 40  # end-to-end steps (each ~1 ms)
# calls in flight in the main measurements (value, e2e, learned): with two, call k+2 is enqueued only after call k's
# rows are read, and the GPU idles on the host between calls; a third keeps one call queued
IN_FLIGHT = 3


def e2e_pipelined(ctxs, streams, h_batches, steps, net=None):
    """`steps` calls of the asynchronous host-buffer localization
    (qcs_loc_localize_async, or qcs_learned_localize_async with net) over the
    contexts used in turn, each on its stream: call k's record copy and row
    copy overlap the kernels of the calls before it, and up to len(ctxs) calls
    are in flight.  Every call copies its pinned records in and its rows and
    counters out; qcs_loc_finish waits for it.  Returns (seconds, rows read)."""
    import torch
    depth = len(ctxs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rows = 0
    for k in range(steps):
        c = ctxs[k % depth]
        if k >= depth:
            rows += c.finish(copy=False)[0].shape[0]
        c.localize_async(h_batches[k % len(h_batches)].data_ptr(), N_PER_STEP,
                         stream=streams[k % len(streams)].cuda_stream, net=net, iters=LEARNED_ITERS,
                         bisections=LEARNED_BISECTIONS)
    for k in range(max(0, steps - depth), steps):
        rows += ctxs[k % depth].finish(copy=False)[0].shape[0]
    return time.perf_counter() - t0, rows


def fit_accuracy(rows, rec, truth, sel, para):
    """Position RMSE (px, per axis), relative photon RMSE and CRLB (px) over sel."""
    fx = rows[sel, 1] + R // 2 - rec[sel, R * R].astype(np.float64)
    fy = rows[sel, 2] + R // 2 - rec[sel, R * R + 1].astype(np.float64)
    rmse = float(np.sqrt(np.mean((fx - truth["x"][sel]) ** 2 + (fy - truth["y"][sel]) ** 2) / 2))
    ph = float(np.sqrt(np.mean((rows[sel, 6] / truth["photons"][sel] - 1) ** 2)))
    crlb = float(np.sqrt(np.mean((rows[sel, 9] ** 2 + rows[sel, 10] ** 2) / 2)) / para.PixelSize)
    return rmse, ph, crlb


def learned_measure(args, streams, ctxs, para, d_batches, h_batches, rec0, truth0, plain_value, world, dist):
    """Learned start points + LEARNED_ITERS BFGS iterations (LEARNED_BISECTIONS
    line-search steps each, analytic gradient) + plain refits of
    the fits the deviance judge rejects + CRLB (qcs_learned_localize_device),
    on the same device-resident batches as the plain step, WLE pre-pass
    included; accuracy of plain vs learned on batch 0 against ground truth."""
    from qcstorm_b200 import lib
    stream, ctx = streams[0], ctxs[0]
    sh = stream.cuda_stream
    net, train = train_learned_net(para, stream)
    # the iteration cap the tuner picks on these records (informational; the timed schedule is fixed)
    tuned_schedule = net.autotune(ctx, d_batches[0].data_ptr(), N_PER_STEP, stream=sh)

    def step(k, s, c=None):
        net.localize(c or ctxs[k % len(ctxs)], d_batches[k % BATCHES].data_ptr(), N_PER_STEP, 0, iters=LEARNED_ITERS,
                     bisections=LEARNED_BISECTIONS, stream=s.cuda_stream)

    ms, windows = device_timed_windows(args.steps, args.warmup, step, streams, dist)
    value = job_rate(args.steps, N_PER_STEP, world, ms)
    one_steps = min(args.steps, 200)
    ms1 = device_timed(one_steps, 3, lambda k, s: step(k, s, ctx), [stream], dist)
    value1 = job_rate(one_steps, N_PER_STEP, world, ms1)

    # accuracy on batch 0: plain and learned rows of the same records
    ctx.localize_device(d_batches[0].data_ptr(), N_PER_STEP, 0, sh)
    plain, _ = ctx.read_rows(sh)
    step(0, stream, ctx)
    learned, _ = ctx.read_rows(sh)
    refits = net.refits(ctx)
    acc_p, acc_l = plain[:, 0] > 0, learned[:, 0] > 0
    both = acc_p & acc_l
    rp, pp, crlb = fit_accuracy(plain, rec0, truth0, both, para)
    rl, pl, _ = fit_accuracy(learned, rec0, truth0, both, para)
    # each arm over its own accepted records (learned accepts more)
    rp_own, pp_own, crlb_p_own = fit_accuracy(plain, rec0, truth0, acc_p, para)
    rl_own, pl_own, crlb_l_own = fit_accuracy(learned, rec0, truth0, acc_l, para)
    # the FP64 Fisher-matrix bound of each arm's own rows (emitters at their fitted positions)
    fisher = {}
    for name, rows in (("plain", plain), ("learned", learned)):
        f = lib.crlb_fisher(para, rows[:N_PER_STEP], rec0)
        sel = (rows[:N_PER_STEP, 0] > 0) & (f[:, 7] == 0)
        rmse, _, _ = fit_accuracy(rows, rec0, truth0, sel, para)
        bound = float(np.sqrt(np.mean((f[sel, 0] ** 2 + f[sel, 1] ** 2) / 2)) / para.PixelSize)
        # each record's error over its own bound: arms that accept different records compare fairly
        ex = rows[sel, 1] + R // 2 - rec0[sel, R * R].astype(np.float64) - truth0["x"][sel]
        ey = rows[sel, 2] + R // 2 - rec0[sel, R * R + 1].astype(np.float64) - truth0["y"][sel]
        norm = float(np.sqrt(np.mean(((ex / f[sel, 0]) ** 2 + (ey / f[sel, 1]) ** 2) / 2) * para.PixelSize ** 2))
        fisher[name] = {"rmse_px": rmse, "crlb_px": bound, "rmse_over_crlb": rmse / bound,
                        "rms_error_over_own_crlb": norm, "rows": int(sel.sum())}
    fisher["learned_minus_plain_rmse_over_crlb"] = (fisher["learned"]["rmse_px"] - fisher["plain"]["rmse_px"]) / \
        fisher["plain"]["crlb_px"]
    fisher["equal_rmse_within_2pct_of_crlb"] = bool(
        fisher["learned"]["rms_error_over_own_crlb"] <= 1.02 * fisher["plain"]["rms_error_over_own_crlb"])
    fisher["basis"] = ("each arm's accepted rows; CRLB = qcs_crlb_fisher_fp64 (full Fisher matrix of the fitted "
                       "model on the ROI's pixels, FP64), per axis; rms_error_over_own_crlb = sqrt(mean((error / "
                       "that record's bound)^2)), the criterion of equal_rmse_within_2pct_of_crlb (learned accepts "
                       "more, harder records, which raise its plain RMSE over its own accepted set)")

    # end to end: pinned host records in, rows out, through qcs_learned_localize_async
    e2e_pipelined(ctxs, streams, h_batches, 4, net=net)
    e2e_steps = E2E_STEPS
    e2e_s, _ = e2e_pipelined(ctxs, streams, h_batches, e2e_steps, net=net)
    e2e_s = max_over_ranks(e2e_s * 1e3, dist) * 1e-3
    start_ms = start_point_ms(net, para, d_batches, stream, dist)
    # the same call without the plain refits of the rejected or poor learned fits (qcs_learned_set_single_refits)
    net.set_single_refits(False)
    nr_steps = min(args.steps, 200)
    ms_nr = device_timed(nr_steps, 3, step, streams, dist)
    step(0, stream, ctx)
    rows_nr, _ = ctx.read_rows(sh)
    net.set_single_refits(True)
    acc_nr = rows_nr[:, 0] > 0
    both_nr = acc_p & acc_nr
    rp_nr, _, _ = fit_accuracy(plain, rec0, truth0, both_nr, para)
    rn, pn, _ = fit_accuracy(rows_nr, rec0, truth0, both_nr, para)
    rn_own, _, _ = fit_accuracy(rows_nr, rec0, truth0, acc_nr, para)
    no_refit = {"value": job_rate(nr_steps, N_PER_STEP, world, ms_nr), "unit": UNIT,
                "vs_plain": job_rate(nr_steps, N_PER_STEP, world, ms_nr) / plain_value,
                "rmse_px": {"plain": rp_nr, "no_refit": rn}, "photon_rel_rmse_no_refit": pn,
                "rmse_px_own_accepted": rn_own, "accepted": float(acc_nr.mean()),
                "basis": "batch 0; records accepted by both plain and this variant (own: its own accepted records)",
                "call": "qcs_learned_set_single_refits(net, 0): the learned fits' results stand"}
    net.close()
    conv = conv_arm(args, streams, ctxs, para, d_batches, rec0, truth0, plain_value, value, start_ms, world, dist)
    return {
        "value": value, "unit": UNIT, "ms_per_step": ms / args.steps, "vs_plain": value / plain_value,
        "windows": windows,
        "value_one_stream": value1, "timing": "three contexts in turn on three streams (value_one_stream: one)",
        "iters": LEARNED_ITERS, "bisections": LEARNED_BISECTIONS, "refits_per_step": refits,
        "autotuned_schedule": {"iters": tuned_schedule[0], "bisections": tuned_schedule[1],
                               "rule": "qcs_learned_autotune: fastest schedule with acceptance within 0.5 points of "
                                       "the best"},
        # mlp_tc (features + network), WLE (5), fit_learned, flag_queue, group refit, refit CRLB, counters, CRLB
        "gpu_launches_per_step": 12,
        "e2e": {"value": e2e_steps * N_PER_STEP * world / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": N_PER_STEP * R * (R + 1) * 2,
                "d2h_bytes_per_step": N_PER_STEP * 48 + 32,
                "call": "qcs_learned_localize_async + qcs_loc_finish on three contexts in turn (pinned records in, "
                        "rows and counters out every step)"},
        "accuracy": {"records": N_PER_STEP, "compared": int(both.sum()),
                     "rmse_px": {"plain": rp, "learned": rl}, "photon_rel_rmse": {"plain": pp, "learned": pl},
                     "crlb_px": crlb, "accepted": {"plain": float((plain[:, 0] > 0).mean()),
                                                   "learned": float((learned[:, 0] > 0).mean())},
                     "equal_rmse": bool(rl <= 1.02 * rp),
                     "basis": "records accepted by both; ground truth of the generator",
                     "fisher_crlb": fisher,
                     "own_accepted": {"rmse_px": {"plain": rp_own, "learned": rl_own},
                                      "photon_rel_rmse": {"plain": pp_own, "learned": pl_own},
                                      "crlb_px": {"plain": crlb_p_own, "learned": crlb_l_own},
                                      "basis": "each arm over the records it accepts"}},
        "train": train,
        "network": "64-128-128-8 MLP on the 7x7 pixels (+2 scale features), BF16 operands, FP32 accumulation; "
                   "inference fused with the features in one tcgen05 kernel",
        "start_points_ms_per_step": start_ms,
        "no_refit": no_refit,
        "conv": conv,
    }


def start_point_ms(net, para, d_batches, stream, dist, steps=20):
    """Device time of the start points alone (network inference) per
    N_PER_STEP-record step."""
    import torch
    st = torch.empty((N_PER_STEP, 5), dtype=torch.float32, device="cuda")
    work = torch.empty((N_PER_STEP * 200,), dtype=torch.float32, device="cuda")
    from qcstorm_b200 import lib
    import ctypes as C

    def step(k, s):
        lib.check(lib.load().qcs_learned_start_device(net.h, C.byref(para), C.c_void_p(d_batches[k % BATCHES].data_ptr()),
                                                      N_PER_STEP, C.c_void_p(st.data_ptr()), C.c_void_p(work.data_ptr()),
                                                      C.c_void_p(s.cuda_stream)))
    return device_timed(steps, 3, step, [stream], dist) / steps


def conv_arm(args, streams, ctxs, para, d_batches, rec0, truth0, plain_value, mlp_value, mlp_start_ms, world, dist):
    """The convolutional start-point network (3x3 conv 32 -> 3x3 conv 64 ->
    FC 256 -> the same outputs; qcs_learned_create_arch(QCS_LEARNED_ARCH_CONV))
    trained on the same records and timed on the same batches with the same
    schedule as the MLP: fits/s, start-point time and accuracy."""
    stream, ctx = streams[0], ctxs[0]
    sh = stream.cuda_stream
    net, train = train_learned_net(para, stream, arch="conv", lr=1e-3)

    def step(k, s, c=None):
        net.localize(c or ctxs[k % len(ctxs)], d_batches[k % BATCHES].data_ptr(), N_PER_STEP, 0, iters=LEARNED_ITERS,
                     bisections=LEARNED_BISECTIONS, stream=s.cuda_stream)

    steps = min(args.steps, 200)
    ms = device_timed(steps, 3, step, streams, dist)
    value = job_rate(steps, N_PER_STEP, world, ms)
    start_ms = start_point_ms(net, para, d_batches, stream, dist)
    ctx.localize_device(d_batches[0].data_ptr(), N_PER_STEP, 0, sh)
    plain, _ = ctx.read_rows(sh)
    step(0, stream, ctx)
    rows, _ = ctx.read_rows(sh)
    refits = net.refits(ctx)
    net.fused_status()
    net.close()
    acc_p, acc_c = plain[:, 0] > 0, rows[:, 0] > 0
    both = acc_p & acc_c
    rp, pp, _ = fit_accuracy(plain, rec0, truth0, both, para)
    rc, pc, _ = fit_accuracy(rows, rec0, truth0, both, para)
    rc_own, _, _ = fit_accuracy(rows, rec0, truth0, acc_c, para)
    return {"value": value, "unit": UNIT, "vs_plain": value / plain_value, "vs_mlp": value / mlp_value,
            "steps": steps, "start_points_ms_per_step": start_ms, "mlp_start_points_ms_per_step": mlp_start_ms,
            "iters": LEARNED_ITERS, "bisections": LEARNED_BISECTIONS, "refits_per_step": refits,
            "accuracy": {"rmse_px": {"plain": rp, "conv": rc}, "photon_rel_rmse": {"plain": pp, "conv": pc},
                         "rmse_px_own_accepted": rc_own, "accepted": {"plain": float(acc_p.mean()),
                                                                      "conv": float(acc_c.mean())},
                         "basis": "batch 0; records accepted by both (own_accepted: the conv arm's own)"},
            "train": train,
            "flops_per_record": 2 * (49 * 9 * 32 + 49 * 288 * 64 + (49 * 64 + 2) * 256 + 256 * 8),
            "network": "conv 3x3x32 -> conv 3x3x64 -> FC 256 -> 8 outputs on the 7x7 pixels (+2 scale features into "
                       "FC), BF16 operands, FP32 accumulation; inference: conv_tc_kernel (padded-grid implicit GEMM, "
                       "tcgen05) + fc_tc_kernel (bulk-copy ring, tcgen05)",
            "default": "mlp (the faster of the two at equal schedule and accuracy)"}


SHAPE_RECORDS = 100_000    # records per call of the other learned workloads
SHAPE_TRAIN = 200_000
SHAPE_STEPS = 20


def emitter_confusion(rows, truth, n, first_frame=1):
    """Localizations per record (its own row, plus an appended second
    emitter) against the generator's emitter count: 3 x 3 counts."""
    count = (rows[:n, 0] > 0).astype(np.int64)
    extra = rows[n:, 11].astype(np.int64) - first_frame
    count[extra[(extra >= 0) & (extra < n)]] += 1
    conf = np.zeros((3, 3), np.int64)
    np.add.at(conf, (truth["k"] - 1, np.minimum(count, 2)), 1)
    return conf.tolist()


def multi_truth_match(rows, rec, truth, R, first_frame=1):
    """Each localization's distance (px) to the nearest true emitter of its
    record (record = frame - first_frame), in ROI coordinates."""
    rows = rows[rows[:, 0] > 0]
    rid = rows[:, 11].astype(np.int64) - first_frame
    fx = rows[:, 1] - rec[rid, R * R].astype(np.float64) + R // 2
    fy = rows[:, 2] - rec[rid, R * R + 1].astype(np.float64) + R // 2
    dx = truth["x"][rid] - fx[:, None]
    dy = truth["y"][rid] - fy[:, None]
    d = np.sqrt(np.nanmin(dx * dx + dy * dy, axis=1))
    ok = d < 1.0
    return {"localizations": int(rows.shape[0]), "matched": int(ok.sum()),
            "rmse_px": float(np.sqrt(np.mean(d[ok] ** 2)))}


def shape_accuracy(kind, plain, learned, rec, truth, R):
    """Plain against learned on the same records: AS3D x/y (px) and z (nm)
    RMSE over the records both accept; multi-emitter localizations within
    1 px of a true emitter and their RMSE."""
    if kind == "multi":
        return {"plain": multi_truth_match(plain, rec, truth, R), "learned": multi_truth_match(learned, rec, truth, R),
                "basis": "localizations within 1 px of a true emitter of their record"}
    both = (plain[:, 0] > 0) & (learned[:, 0] > 0)

    def rm(rows):
        fx = rows[both, 1] + R // 2 - rec[both, R * R].astype(np.float64)
        fy = rows[both, 2] + R // 2 - rec[both, R * R + 1].astype(np.float64)
        xy = float(np.sqrt(np.mean((fx - truth["x"][both]) ** 2 + (fy - truth["y"][both]) ** 2) / 2))
        z = float(np.sqrt(np.mean((rows[both, 3] - truth["z"][both]) ** 2)))
        return {"rmse_px": xy, "z_rmse_nm": z, "accepted": float((rows[:, 0] > 0).mean())}
    return {"plain": rm(plain), "learned": rm(learned), "compared": int(both.sum()),
            "basis": "records accepted by both; ground truth of the generator"}


TWO_ITERS = 3  # BFGS iterations of the learned-start two-emitter fits (6 line-search steps)


def train_two_emitter_net(ctx_tr, para, d_tr, feat, scale, n, R, epochs, stream):
    """A two-emitter start-point network trained on the records whose plain
    two-emitter fit (the plain multi-emitter call just made on ctx_tr) kept
    both emitters."""
    from qcstorm_b200 import lib
    t2, v2 = lib.two_emitter_targets(ctx_tr, para, d_tr.data_ptr(), scale, n, stream.cuda_stream)
    stream.synchronize()
    net2 = lib.LearnedNet(batch=4096, seed=6, loc_type=lib.LEARNED_GS2D_2E, roi_size=R)
    net2.train(feat, t2, v2, epochs=epochs, lr=2e-3, stream=stream.cuda_stream)
    stream.synchronize()
    return net2


def train_three_emitter_net(ctx_tr, para, d_tr, feat, scale, n, R, epochs, stream):
    """A three-emitter start-point network trained on the parameters the
    plain three-emitter fit converged to (captured in the plain call just made
    on ctx_tr) for the records where it kept an emitter."""
    from qcstorm_b200 import lib
    t3, v3 = lib.three_emitter_targets(ctx_tr, para, d_tr.data_ptr(), scale, n, stream.cuda_stream)
    stream.synchronize()
    net3 = lib.LearnedNet(batch=4096, seed=7, loc_type=lib.LEARNED_GS2D_3E, roi_size=R)
    net3.train(feat, t3, v3, epochs=epochs, lr=2e-3, stream=stream.cuda_stream)
    stream.synchronize()
    return net3


THREE_ITERS = 4  # three-emitter fits from the network's start points: 4 x 6 (plain 16 x 11)


def learned_shapes_measure(streams, dist, world, rank, mufu_peak=None, cpu_baseline=True):
    """The learned path on the other configurations' generators, each against
    plain fitting of the same device-resident records with two contexts in
    turn: astigmatic 3D 9x9 ROIs (single-emitter fits from sigma_x / sigma_y
    start points, 3 iterations of 6 line-search steps against the reference's
    11 of 11) and 1-3 emitter 11x11 ROIs with multi-emitter fitting (learned
    single-emitter stage, 2 x 6, and emitter-count classes routing records
    straight to the 2E / 3E fits).  Networks trained on the GPU on
    SHAPE_TRAIN records of other seeds labelled by plain fitting."""
    import torch
    from qcstorm_b200 import lib, synth
    s0 = streams[0]
    sh = s0.cuda_stream
    out = {}
    for kind, gen, R, iters, bis in (("as3d", synth.as3d_rois, 9, 3, 6), ("multi", synth.multi_rois, 11, 2, 6)):
        t0 = time.perf_counter()
        tr, para, _ = gen(SHAPE_TRAIN, R=R, seed=7000 + 10 * rank)
        d_tr = torch.from_numpy(tr.view(np.int16)).cuda()
        ctx_tr = lib.LocContext(para, capacity=SHAPE_TRAIN)
        if kind == "multi":
            lib.set_three_emitter_capture(ctx_tr)  # the three-emitter network's targets
        ctx_tr.localize_device(d_tr.data_ptr(), SHAPE_TRAIN, 0, sh)
        labels = lib.count_labels(ctx_tr, SHAPE_TRAIN, sh) if kind == "multi" else None
        feat, scale = lib.LearnedNet.features(para, d_tr.data_ptr(), SHAPE_TRAIN, stream=sh)
        tgt, valid = lib.LearnedNet.targets(para, d_tr.data_ptr(), ctx_tr.device_rows(), scale, SHAPE_TRAIN,
                                            stream=sh)
        s0.synchronize()
        if labels is not None:
            valid = valid * (labels == 0).float()
        torch.cuda.synchronize()
        net = lib.LearnedNet(batch=4096, seed=5, loc_type=para.LocType, roi_size=R)
        net.train(feat, tgt, valid, epochs=TRAIN_EPOCHS, lr=2e-3, stream=sh, classes=labels)
        net2 = net3 = None
        if kind == "multi":
            net.set_count_threshold(0.5)
            net2 = train_two_emitter_net(ctx_tr, para, d_tr, feat, scale, SHAPE_TRAIN, R, TRAIN_EPOCHS, s0)
            net3 = train_three_emitter_net(ctx_tr, para, d_tr, feat, scale, SHAPE_TRAIN, R, TRAIN_EPOCHS, s0)
        torch.cuda.synchronize()
        ctx_tr.close()
        del d_tr, feat, scale, tgt, valid, labels
        train_s = time.perf_counter() - t0

        recs, truths, d_b = [], [], []
        for b in range(2):
            rec, _, truth = gen(SHAPE_RECORDS, R=R, seed=8000 + 10 * rank + b)
            recs.append(rec)
            truths.append(truth)
            d_b.append(torch.from_numpy(rec.view(np.int16)).cuda())
        ctxs = [lib.LocContext(para, capacity=SHAPE_RECORDS) for _ in range(len(streams))]

        def plain(k, s, c=None):
            (c or ctxs[k % len(ctxs)]).localize_device(d_b[k % 2].data_ptr(), SHAPE_RECORDS, 0, s.cuda_stream)

        def learned(k, s, c=None):
            net.localize(c or ctxs[k % len(ctxs)], d_b[k % 2].data_ptr(), SHAPE_RECORDS, iters=iters, bisections=bis,
                         stream=s.cuda_stream)

        ms_p = device_timed(SHAPE_STEPS, 3, plain, streams, dist)
        ms_l = device_timed(SHAPE_STEPS, 3, learned, streams, dist)
        plain(0, s0, ctxs[0])
        rows_p, ratios_p = ctxs[0].read_rows(sh)
        # roofline of the plain call: MUFU operations of its fits (reference schedule) over its time, and
        # its single-emitter stage's kernel alone (the dominant kernel) on the same records
        roof = None
        if mufu_peak:
            n = SHAPE_RECORDS
            single = int(round(float(ratios_p[0]) * n))
            n2, n3 = int(round(float(ratios_p[1]) * n)), int(round(float(ratios_p[2]) * n))
            ops = cascade_mufu_ops(R, single, n2, n3, single_kind="as3d" if kind == "as3d" else "gs2d")
            call_ms = ms_p / SHAPE_STEPS
            wle_b = torch.empty((n, 6), dtype=torch.float32, device="cuda")
            lib.check(lib.load().qcs_wle_estimate_device(ctxs[0].h, C.c_void_p(d_b[0].data_ptr()), n, C.byref(para),
                                                         C.c_void_p(wle_b.data_ptr()), C.c_void_p(sh)))
            d_loc = torch.empty((n, 12), dtype=torch.float32, device="cuda")
            for _ in range(2):
                lib.fit_single_device(para.LocType, para, d_b[0].data_ptr(), wle_b.data_ptr(), n, d_loc.data_ptr(), sh)
            kt = []
            for _ in range(10):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(s0)
                lib.fit_single_device(para.LocType, para, d_b[0].data_ptr(), wle_b.data_ptr(), n, d_loc.data_ptr(),
                                      sh)
                b.record(s0)
                kt.append((a, b))
            torch.cuda.synchronize()
            k_ms = statistics.mean(a.elapsed_time(b) for a, b in kt)
            k_ops = cascade_mufu_ops(R, n, single_kind="as3d" if kind == "as3d" else "gs2d")
            roof = {"bound": "sfu", "unit": "MUFU op/s", "peak": mufu_peak,
                    "call": {"achieved": ops / (call_ms * 1e-3), "frac": ops / (call_ms * 1e-3) / mufu_peak,
                             "ms": call_ms, "stages": {"single": single, "two_emitter": n2, "three_emitter": n3},
                             "scope": "whole plain call (WLE + fit cascade + CRLB), three contexts in turn; fits counted "
                                      "on the reference schedule"},
                    "kernel": {"name": "fit_single_kernel<%d,%s>" % (R, "AS3D" if kind == "as3d" else "GS2D"),
                               "achieved": k_ops / (k_ms * 1e-3), "frac": k_ops / (k_ms * 1e-3) / mufu_peak,
                               "ms": k_ms, "records": n}}
            del wle_b, d_loc
        learned(0, s0, ctxs[0])
        rows_l, ratios_l = ctxs[0].read_rows(sh)
        refits = net.refits(ctxs[0])
        net.fused_status()
        two = None
        if net2 is not None:
            net.set_two_emitter(net2, iters=TWO_ITERS, bisections=6)
            ms_l2 = device_timed(SHAPE_STEPS, 3, learned, streams, dist)
            learned(0, s0, ctxs[0])
            rows_l2, _ = ctxs[0].read_rows(sh)
            two = {"learned_fits_per_s": job_rate(SHAPE_STEPS, SHAPE_RECORDS, world, ms_l2), "vs_plain": ms_p / ms_l2,
                   "schedule": "two-emitter fits from the network's start points, %d x 6 (plain: 13 x 11); poor ones "
                               "on to the three-emitter fit" % TWO_ITERS,
                   "accuracy": multi_truth_match(rows_l2, recs[0], truths[0], R)}
            net.set_two_emitter(net2, iters=TWO_ITERS, bisections=6, fallback="plain")
            ms_l3 = device_timed(SHAPE_STEPS, 3, learned, streams, dist)
            learned(0, s0, ctxs[0])
            rows_l3, _ = ctxs[0].read_rows(sh)
            two["plain_refit"] = {"learned_fits_per_s": job_rate(SHAPE_STEPS, SHAPE_RECORDS, world, ms_l3),
                                  "two_emitter_refits_per_call": net.refits_2e(ctxs[0]),
                                  "accuracy": multi_truth_match(rows_l3, recs[0], truths[0], R)}
            # and the three-emitter fits from their network's start points (QCS_LEARNED_GS2D_3E)
            three = {"schedule": "three-emitter fits from the network's start points, %d x 6 (plain: 16 x 11); poor "
                                 "ones refitted plainly" % THREE_ITERS}
            for fb, th, direct in (("3e", 0.0, False), ("plain", 0.0, False), ("plain", -1.0, False),
                                   ("none", -1.0, False), ("plain", -1.0, True), ("none", -1.0, True)):
                net.set_two_emitter(net2, iters=TWO_ITERS, bisections=6, fallback=fb)
                net.set_three_emitter(net3, iters=THREE_ITERS, bisections=6, dev_th=th)
                net.set_direct_two_emitter(direct)
                ms_t = device_timed(SHAPE_STEPS, 3, learned, streams, dist)
                learned(0, s0, ctxs[0])
                rows_t, _ = ctxs[0].read_rows(sh)
                net.set_direct_two_emitter(False)
                three["two_emitter_fallback_" + fb + ("_no_3e_refits" if th < 0 else "") +
                      ("_direct_two_emitter" if direct else "")] = {
                    "learned_fits_per_s": job_rate(SHAPE_STEPS, SHAPE_RECORDS, world, ms_t), "vs_plain": ms_p / ms_t,
                    "two_emitter_refits_per_call": net.refits_2e(ctxs[0]),
                    "three_emitter_refits_per_call": net.refits_3e(ctxs[0]),
                    "accuracy": multi_truth_match(rows_t, recs[0], truths[0], R)}
            net.set_three_emitter(None)
            net3.close()
            two["with_three_emitter_starts"] = three
            net.set_two_emitter(None)
            net2.close()
            # poor bright single fits straight to the two-emitter fit (no plain refit first)
            net.set_direct_two_emitter(True)
            ms_d = device_timed(SHAPE_STEPS, 3, learned, streams, dist)
            learned(0, s0, ctxs[0])
            rows_d, _ = ctxs[0].read_rows(sh)
            net.set_direct_two_emitter(False)
            two["direct_two_emitter"] = {"learned_fits_per_s": job_rate(SHAPE_STEPS, SHAPE_RECORDS, world, ms_d),
                                         "vs_plain": ms_p / ms_d,
                                         "accuracy": multi_truth_match(rows_d, recs[0], truths[0], R),
                                         "note": "without the two-emitter starts; qcs_learned_set_direct_two_emitter"}
        out[kind] = {
            "workload": ("astigmatic 3D 9x9 ROIs, z U(-600,600) nm, photons log-U[1000,8000], background U(20,150), "
                         "camera ADU (offset 100, 0.45 e-/ADU)" if kind == "as3d" else
                         "11x11 ROIs with 1/2/3 emitters (p 0.5/0.3/0.2) 1-3 px apart, multi-emitter fitting on"),
            "records_per_call": SHAPE_RECORDS,
            "plain_fits_per_s": job_rate(SHAPE_STEPS, SHAPE_RECORDS, world, ms_p),
            "learned_fits_per_s": job_rate(SHAPE_STEPS, SHAPE_RECORDS, world, ms_l),
            "vs_plain": ms_p / ms_l,
            "schedule": "%d BFGS iterations x %d line-search steps (plain: the reference's %s)" % (
                iters, bis, "11 x 11" if kind == "as3d" else "8 x 11 single, 13 x 11 2E, 16 x 11 3E"),
            "refits_per_call": refits,
            "single_emitter_fits_per_call": {"plain": int(round(float(ratios_p[0]) * SHAPE_RECORDS)),
                                             "learned": int(round(float(ratios_l[0]) * SHAPE_RECORDS))},
            "accuracy": shape_accuracy(kind, rows_p, rows_l, recs[0], truths[0], R),
            "train": {"records": SHAPE_TRAIN, "epochs": TRAIN_EPOCHS, "seconds": train_s},
        }
        if two is not None:
            out[kind]["with_two_emitter_starts"] = two
        if roof is not None:
            out[kind]["plain_roofline"] = roof
        if kind == "multi":
            # the FP64 likelihood-ratio model selection on the same records, against the reference's cascade:
            # fits/s and localizations per record against the generator's emitter count
            for c in ctxs:
                c.set_model_selection("lr")
            lr_th = ctxs[0].model_selection()[1]
            ms_lr = device_timed(SHAPE_STEPS, 3, plain, streams, dist)
            plain(0, s0, ctxs[0])
            rows_lr, ratios_lr = ctxs[0].read_rows(sh)
            for c in ctxs:
                c.set_model_selection("cascade")
            out[kind]["lr_selection"] = {
                "fits_per_s": job_rate(SHAPE_STEPS, SHAPE_RECORDS, world, ms_lr), "vs_cascade": ms_p / ms_lr,
                "threshold": lr_th,
                "kept_1_2_3_emitters": [float(x) for x in ratios_lr[3:6]],
                "localizations_per_record_by_true_count": {
                    "cascade": emitter_confusion(rows_p, truths[0], SHAPE_RECORDS),
                    "lr": emitter_confusion(rows_lr, truths[0], SHAPE_RECORDS)},
                "accuracy": {"cascade": multi_truth_match(rows_p, recs[0], truths[0], R),
                             "lr": multi_truth_match(rows_lr, recs[0], truths[0], R)},
                "basis": "rows: true emitters 1..3, columns: localizations 0..2 (at most two per record, as the "
                         "reference writes them)"}
        if cpu_baseline and rank == 0:
            out[kind]["cpu_baseline"] = shape_cpu_baseline(kind, R, 1500 if kind == "as3d" else 600)
        for c in ctxs:
            c.close()
        net.close()
    return out


MIXED_TRAIN = 4_000_000    # training records of the mixed 7/9/11 workload (all three shapes)
MIXED_EVAL = 10_000_000    # fresh evaluation records of it
MIXED_CALL = 100_000       # records per localization call
MIXED_EPOCHS = 2
# (generator, ROI size, learned BFGS iterations, line-search steps)
MIXED_SHAPES = (("gs2d", 7, 2, 6), ("as3d", 9, 3, 6), ("multi", 11, 2, 6))


def _split(total, parts):
    return [total // parts + (1 if i < total % parts else 0) for i in range(parts)]


class _SingleAcc:
    """Sums over calls for single-emitter shapes: position error (px), z error
    (nm) and CRLB (px) over the records both modes accept."""

    def __init__(self):
        self.n = 0
        self.se = {"plain": 0.0, "learned": 0.0}
        self.sz = {"plain": 0.0, "learned": 0.0}
        self.crlb = {"plain": 0.0, "learned": 0.0}
        self.crlb_n = {"plain": 0, "learned": 0}
        self.acc = {"plain": 0, "learned": 0}
        self.total = 0

    def add(self, rows, truth, o, R, pixel_nm):
        rp, rl = rows["plain"], rows["learned"]
        m = rp.shape[0]
        both = (rp[:, 0] > 0) & (rl[:, 0] > 0)
        self.n += int(both.sum())
        self.total += m
        tx, ty = truth["x"][o:o + m][both], truth["y"][o:o + m][both]
        for mode, r in rows.items():
            self.acc[mode] += int((r[:, 0] > 0).sum())
            fx = r[both, 1].astype(np.float64) + R // 2 - 1024
            fy = r[both, 2].astype(np.float64) + R // 2 - 1024
            self.se[mode] += float(np.sum((fx - tx) ** 2 + (fy - ty) ** 2) / 2)
            if "z" in truth:
                self.sz[mode] += float(np.sum((r[both, 3].astype(np.float64) - truth["z"][o:o + m][both]) ** 2))
            c = r[both, 9:11].astype(np.float64) / pixel_nm
            c2 = (c[:, 0] ** 2 + c[:, 1] ** 2) / 2
            fin = np.isfinite(c2)
            self.crlb[mode] += float(np.sum(c2[fin]))
            self.crlb_n[mode] += int(fin.sum())

    def result(self, has_z):
        out = {}
        for mode in ("plain", "learned"):
            d = {"rmse_px": math.sqrt(self.se[mode] / max(self.n, 1)),
                 "crlb_px": math.sqrt(self.crlb[mode] / max(self.crlb_n[mode], 1)),
                 "crlb_not_finite": self.n - self.crlb_n[mode],
                 "accepted": self.acc[mode] / max(self.total, 1)}
            if has_z:
                d["z_rmse_nm"] = math.sqrt(self.sz[mode] / max(self.n, 1))
            d["rmse_over_crlb"] = d["rmse_px"] / d["crlb_px"] if d["crlb_px"] > 0 else None
            out[mode] = d
        out["compared"] = self.n
        out["basis"] = "records accepted by both; ground truth of the generator; CRLB = the rows' own (cols 9-10, finite ones)"
        return out


class _MultiAcc:
    """Sums over calls for multi-emitter ROIs: localizations within 1 px of a
    true emitter of their record, their squared distances."""

    def __init__(self):
        self.loc = {"plain": 0, "learned": 0}
        self.hit = {"plain": 0, "learned": 0}
        self.se = {"plain": 0.0, "learned": 0.0}

    def add(self, rows, truth, o, R, pixel_nm):
        for mode, r in rows.items():
            r = r[r[:, 0] > 0]
            rid = r[:, 11].astype(np.int64) - 1
            fx = r[:, 1].astype(np.float64) + R // 2 - 1024
            fy = r[:, 2].astype(np.float64) + R // 2 - 1024
            dx = truth["x"][rid] - fx[:, None]
            dy = truth["y"][rid] - fy[:, None]
            d2 = np.nanmin(dx * dx + dy * dy, axis=1)
            ok = d2 < 1.0
            self.loc[mode] += int(r.shape[0])
            self.hit[mode] += int(ok.sum())
            self.se[mode] += float(d2[ok].sum())

    def result(self, has_z):
        out = {mode: {"localizations": self.loc[mode], "matched": self.hit[mode],
                      "rmse_px": math.sqrt(self.se[mode] / max(self.hit[mode], 1))} for mode in ("plain", "learned")}
        out["basis"] = "localizations within 1 px of a true emitter of their record"
        return out


def mixed_measure(streams, dist, world, rank):
    """The learned path on the mixed 7x7 / 9x9 / 11x11 workload: the GS2D 7x7,
    astigmatic 3D 9x9 and 1-3 emitter 11x11 generators in equal parts,
    MIXED_TRAIN records (seeded, made on the GPU) labelled by plain fitting
    train one network per ROI size, and MIXED_EVAL fresh records are localized
    in calls of MIXED_CALL records of one size (the reference's API takes one
    ROI size per call) plainly and with learned start points.  fits/s over the
    whole evaluation stream (device time of every call, three contexts in turn),
    accuracy against the generator's truth with the rows' own CRLB beside it."""
    import torch
    from qcstorm_b200 import lib, synth_torch as ST
    s0 = streams[0]
    sh = s0.cuda_stream
    n_train = _split(MIXED_TRAIN, len(MIXED_SHAPES))
    n_eval = _split(MIXED_EVAL, len(MIXED_SHAPES))
    shapes = {}
    tot_p = tot_l = 0.0
    for i, (kind, R, iters, bis) in enumerate(MIXED_SHAPES):
        para = ST.para(kind, R)
        t0 = time.perf_counter()
        d_tr, _ = ST.rois(kind, n_train[i], R, seed=20_000 + 100 * rank + i, device="cuda")
        torch.cuda.synchronize()
        ctx_tr = lib.LocContext(para, capacity=n_train[i])
        if kind == "multi":
            lib.set_three_emitter_capture(ctx_tr)  # the three-emitter network's targets
        ctx_tr.localize_device(d_tr.data_ptr(), n_train[i], 0, sh)
        labels = lib.count_labels(ctx_tr, n_train[i], sh) if kind == "multi" else None
        feat, scale = lib.LearnedNet.features(para, d_tr.data_ptr(), n_train[i], stream=sh)
        tgt, valid = lib.LearnedNet.targets(para, d_tr.data_ptr(), ctx_tr.device_rows(), scale, n_train[i],
                                            stream=sh)
        s0.synchronize()
        if labels is not None:
            valid = valid * (labels == 0).float()
        torch.cuda.synchronize()
        net = lib.LearnedNet(batch=4096, seed=5, loc_type=para.LocType, roi_size=R)
        net.train(feat, tgt, valid, epochs=MIXED_EPOCHS, lr=2e-3, stream=sh, classes=labels)
        net2 = net3 = None
        if kind != "multi":
            net.set_single_refits(False)  # the learned fits' results stand (accuracy below)
        if kind == "multi":
            net.set_count_threshold(0.5)
            net2 = train_two_emitter_net(ctx_tr, para, d_tr, feat, scale, n_train[i], R, MIXED_EPOCHS, s0)
            net3 = train_three_emitter_net(ctx_tr, para, d_tr, feat, scale, n_train[i], R, MIXED_EPOCHS, s0)
            # the fastest variant that beats plain fitting on accuracy: poor bright single fits straight to the
            # two-emitter fit, two- and three-emitter fits from their networks' start points without plain refits
            net.set_two_emitter(net2, iters=TWO_ITERS, bisections=6, fallback="none")
            net.set_three_emitter(net3, iters=THREE_ITERS, bisections=6, dev_th=-1.0)
            net.set_direct_two_emitter(True)
        torch.cuda.synchronize()
        ctx_tr.close()
        del d_tr, feat, scale, tgt, valid, labels
        train_s = time.perf_counter() - t0

        d_ev, truth = ST.rois(kind, n_eval[i], R, seed=30_000 + 100 * rank + i, device="cuda")
        torch.cuda.synchronize()
        rb = R * (R + 1) * 2
        base = d_ev.data_ptr()
        calls = [(o, min(MIXED_CALL, n_eval[i] - o)) for o in range(0, n_eval[i], MIXED_CALL)]
        ctxs = [lib.LocContext(para, capacity=MIXED_CALL) for _ in range(len(streams))]

        def plain(k, s, c=None):
            o, m = calls[k % len(calls)]
            (c or ctxs[k % len(ctxs)]).localize_device(base + o * rb, m, 0, s.cuda_stream)

        def learned(k, s, c=None):
            o, m = calls[k % len(calls)]
            net.localize(c or ctxs[k % len(ctxs)], base + o * rb, m, iters=iters, bisections=bis, stream=s.cuda_stream)

        ms_p = device_timed(len(calls), 3, plain, streams, dist)
        ms_l = device_timed(len(calls), 3, learned, streams, dist)
        tot_p += ms_p
        tot_l += ms_l
        truth_h = {k: v.cpu().numpy() for k, v in truth.items()}
        acc = _MultiAcc() if kind == "multi" else _SingleAcc()
        for k, (o, m) in enumerate(calls):
            rows = {}
            plain(k, s0, ctxs[0])
            rows["plain"] = ctxs[0].read_rows(sh)[0]
            learned(k, s0, ctxs[0])
            rows["learned"] = ctxs[0].read_rows(sh)[0]
            acc.add(rows, truth_h, o, R, para.PixelSize)
        net.fused_status()
        shapes["%s%d" % (kind, R)] = {
            "train_records": n_train[i], "eval_records": n_eval[i], "calls": len(calls),
            "plain_fits_per_s": n_eval[i] * world / (ms_p * 1e-3),
            "learned_fits_per_s": n_eval[i] * world / (ms_l * 1e-3), "vs_plain": ms_p / ms_l,
            "schedule": "learned %d x %d" % (iters, bis) + ("; no plain refits" if kind != "multi" else "") + (
                "; poor bright single fits straight to the two-emitter fit; two-emitter fits from the network's start "
                "points, %d x 6, and three-emitter fits from theirs, %d x 6, without plain refits (more emitters "
                "found than the plain cascade, see accuracy)" % (TWO_ITERS, THREE_ITERS) if net2 else ""),
            "train_seconds": train_s,
            "accuracy": acc.result(kind == "as3d")}
        for c in ctxs:
            c.close()
        if net2 is not None:
            net.set_two_emitter(None)
            net2.close()
        if net3 is not None:
            net.set_three_emitter(None)
            net3.close()
        net.close()
        del d_ev, truth, truth_h
        torch.cuda.empty_cache()
    return {"workload": "GS2D 7x7, astigmatic 3D 9x9 and 1-3 emitter 11x11 ROIs in equal parts (the three "
                        "single-size generators), records made on the GPU from seeds",
            "train_records": MIXED_TRAIN * world, "eval_records": MIXED_EVAL * world, "records_per_call": MIXED_CALL,
            "train_epochs": MIXED_EPOCHS,
            "plain_fits_per_s": MIXED_EVAL * world / (tot_p * 1e-3),
            "learned_fits_per_s": MIXED_EVAL * world / (tot_l * 1e-3), "vs_plain": tot_p / tot_l,
            "timing": "device time of every evaluation call, three contexts in turn, summed over the sizes",
            "shapes": shapes}


def mixed_persistent_measure(streams, dist, world, rank):
    """Plain fitting of the mixed 7/9/11 evaluation stream (mixed_measure's
    records, same seeds) two ways over the same chunks: one
    qcs_loc_localize_mixed_device call per MIXED_CALL records of each size
    (the three sizes' single-emitter fits in one persistent launch), and the
    same chunks as three qcs_loc_localize_device calls in a row.  Device time
    of every call, three sets of contexts in turn; the rows of one chunk are
    compared bit for bit."""
    import torch
    from qcstorm_b200 import lib, synth_torch as ST
    n_eval = _split(MIXED_EVAL, len(MIXED_SHAPES))
    data = []
    for i, (kind, R, _, _) in enumerate(MIXED_SHAPES):
        d_ev, _ = ST.rois(kind, n_eval[i], R, seed=30_000 + 100 * rank + i, device="cuda")
        data.append((R, ST.para(kind, R), d_ev, n_eval[i]))
    torch.cuda.synchronize()
    ncalls = max((n + MIXED_CALL - 1) // MIXED_CALL for _, _, _, n in data)
    ctxs = [[lib.LocContext(para, capacity=MIXED_CALL) for _, para, _, _ in data] for _ in range(len(streams))]

    def chunks(k, cs):
        out = []
        for j, (R, para, d, n) in enumerate(data):
            o = (k % ncalls) * MIXED_CALL
            m = min(MIXED_CALL, n - o)
            if m > 0:
                out.append((cs[j], d.data_ptr() + o * R * (R + 1) * 2, m))
        return out

    def mixed(k, s, cs=None):
        lib.localize_mixed_device(chunks(k, cs or ctxs[k % len(ctxs)]), s.cuda_stream)

    def per_size(k, s, cs=None):
        for c, ptr, m in chunks(k, cs or ctxs[k % len(ctxs)]):
            c.localize_device(ptr, m, 0, s.cuda_stream)

    ms_m = device_timed(ncalls, 3, mixed, streams, dist)
    ms_s = device_timed(ncalls, 3, per_size, streams, dist)
    sh = streams[0].cuda_stream
    # chunk 0 through both paths, one size at a time and all three, one stream
    per_entry = {}
    first = chunks(0, ctxs[0])
    for name, sub in [("R%d" % data[j][0], [first[j]]) for j in range(len(first))] + [("all", first)]:
        t_m = device_timed(5, 2, lambda k, s: lib.localize_mixed_device(sub, s.cuda_stream), streams[:1], dist)
        t_s = device_timed(5, 2, lambda k, s: [c.localize_device(p, m, 0, s.cuda_stream) for c, p, m in sub],
                           streams[:1], dist)
        per_entry[name] = {"persistent_ms": t_m / 5, "per_size_ms": t_s / 5}
    per_size(0, streams[0], ctxs[0])
    base = [c.read_rows(sh)[0] for c in ctxs[0]]
    mixed(0, streams[0], ctxs[0])
    equal = all(np.array_equal(c.read_rows(sh)[0].view(np.uint32), b.view(np.uint32)) for c, b in zip(ctxs[0], base))
    for cs in ctxs:
        for c in cs:
            c.close()
    del data
    torch.cuda.empty_cache()
    return {"workload": "the mixed 7/9/11 evaluation records (GS2D 7x7, astigmatic 3D 9x9, 1-3 emitter 11x11), plain "
                        "fitting, %d records of each size per call" % MIXED_CALL,
            "calls": ncalls, "eval_records": MIXED_EVAL * world,
            "persistent_fits_per_s": MIXED_EVAL * world / (ms_m * 1e-3),
            "per_size_fits_per_s": MIXED_EVAL * world / (ms_s * 1e-3), "persistent_vs_per_size": ms_s / ms_m,
            "rows_equal": bool(equal), "per_entry": per_entry,
            "timing": "device time of every call, three sets of contexts in turn; per_entry: one chunk of each size "
                      "alone and all three, one stream, 5 calls after 2 warm-ups"}


CONSEC_FRAMES_PER_GROUP = 32
CONSEC_GROUPS = 8


def consec_measure(stream, dist, world):
    """Consecutive-frame merging (qcs_consec_fit_device) of localization rows
    of blinking molecules, ~3,000 rows per 2048 x 2048 frame, groups of
    CONSEC_FRAMES_PER_GROUP frames as the plug-ins write them (each call
    merges the previous group with the new one and CRLBs the rows that
    leave): rows/s over CONSEC_GROUPS calls, CUDA events on the call's
    stream (the call synchronizes at its end, as the reference's does)."""
    import torch
    from qcstorm_b200 import lib, synth
    from qcstorm_b200.abi import default_para
    rows, counts = synth.blinking_rows(n_emitters=7500, frames=CONSEC_FRAMES_PER_GROUP * 2, seed=3, width=2048)
    sizes = synth.group_sizes(counts, CONSEC_FRAMES_PER_GROUP)
    para = default_para(LocType=0, ConsecFit_DistanceTh_nm=80.0, PixelSize=100.0, QE=0.72)
    cap = int(sizes.max())
    cf = lib.ConsecFit(capacity=cap)
    d = [torch.from_numpy(rows[o:o + k].copy()).cuda() for o, k in zip(np.r_[0, np.cumsum(sizes)[:-1]], sizes)]
    sh = stream.cuda_stream
    torch.cuda.synchronize()
    for g in range(3):
        cf.fit_device(d[g % 2].data_ptr(), int(sizes[g % 2]), para, stream=sh)
    merged = cf.fit_device(d[1].data_ptr(), int(sizes[1]), para, stream=sh)
    zeroed = int((cf.read_rows()[:, 0] == 0).sum())
    on_ratios = cf.ontime_ratio()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    total = 0
    for g in range(CONSEC_GROUPS):
        cf.fit_device(d[g % 2].data_ptr(), int(sizes[g % 2]), para, stream=sh)
        total += int(sizes[g % 2])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist) / CONSEC_GROUPS
    cf.close()
    # localization statistics (qcs_stat_get_statistical_inf_device) on the same groups
    stt = lib.Statistics(capacity=cap)
    for g in range(2):
        stt.update_device(d[g % 2].data_ptr(), int(sizes[g % 2]), para, stream=sh)
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for g in range(CONSEC_GROUPS):
        _, means = stt.update_device(d[g % 2].data_ptr(), int(sizes[g % 2]), para, stream=sh)
    s1.record(stream)
    torch.cuda.synchronize()
    ms_stat = max_over_ranks(s0.elapsed_time(s1), dist) / CONSEC_GROUPS
    # the on-time fit the plug-ins run after each merge (host arithmetic, as in the reference)
    t0 = time.perf_counter()
    for _ in range(100):
        mean_on, shown = stt.update_ontime(on_ratios)
    us_on = (time.perf_counter() - t0) * 1e4
    stt.close()
    stat = {"rows_per_call": int(total / CONSEC_GROUPS), "ms_per_call": ms_stat,
            "rows_per_s": world * total / (ms_stat * 1e-3 * CONSEC_GROUPS),
            "activation_density_per_um2": float(means[6]), "mean_precision_nm": float(means[1]),
            "ontime_fit": {"mean_ontime_frames": float(mean_on), "ratios_1_2_3_4plus": [float(v) for v in shown[:4]],
                           "us_per_call": us_on, "call": "qcs_stat_update_ontime_ratio (host, 10 ratios)"},
            "call": "qcs_stat_get_statistical_inf_device (histograms, means, activation density over 30 frames)"}
    return {"statistics": stat, "workload": "rows of 7,500 blinking molecules over 2048 x 2048 frames (~%d rows per frame), %d frames "
                        "per call, threshold 80 nm at 100 nm pixels" % (int(counts.mean()), CONSEC_FRAMES_PER_GROUP),
            "rows_per_call": int(total / CONSEC_GROUPS), "ms_per_call": ms,
            "rows_per_s": world * total / (ms * 1e-3 * CONSEC_GROUPS),
            "rows_zeroed_per_call": zeroed, "rows_out_per_call": merged,
            "call": "qcs_consec_fit_device (link by sorted (frame, y) search, merge, remove, CRLB)"}


def autotune_measure(stream, dist, world):
    """The autotuner on small calls: qcs_loc_autotune's table for GS2D 7x7 and
    the device time of 2,000-record calls (WLE pre-pass, fit, CRLB) with and
    without it (the rows are identical)."""
    import torch
    from qcstorm_b200 import lib, synth
    rec, para, _ = synth.gs2d_rois(20_000, R=R, seed=99)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = lib.LocContext(para, capacity=20_000)
    wle = torch.from_numpy(ctx.wle(rec)).cuda()
    sh = stream.cuda_stream
    torch.cuda.synchronize()
    table = ctx.autotune(d.data_ptr(), wle.data_ptr(), 20_000, stream=sh)
    out = {"table": [{"records_up_to": a, "lanes_per_roi": b} for a, b in table]}
    for m in (2000, 20_000):
        res = {}
        for name, tab in (("one_thread_per_roi", []), ("tuned", table)):
            ctx.set_tuning(tab)
            for _ in range(3):
                ctx.localize_device(d.data_ptr(), m, 0, sh)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(20):
                ctx.localize_device(d.data_ptr(), m, 0, sh)
            e1.record(stream)
            torch.cuda.synchronize()
            res[name + "_ms"] = max_over_ranks(e0.elapsed_time(e1), dist) / 20
        out["call_%d_records" % m] = res
    ctx.close()
    # the multi-emitter stages: lane groups against one thread per ROI, by queue length (11x11, 1-3 emitters)
    rec, para, _ = synth.multi_rois(50_000, R=11, seed=98)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = lib.LocContext(para, capacity=50_000)
    wle = torch.from_numpy(ctx.wle(rec)).cuda()
    torch.cuda.synchronize()
    ctx.autotune(d.data_ptr(), wle.data_ptr(), 50_000, stream=sh)
    l2, l3 = ctx.tuning_multi()
    out["multi_emitter_11x11"] = {"lane_group_queue_limit_2e": l2, "lane_group_queue_limit_3e": l3,
                                  "note": "longest stage queue for which the lane-group kernel beat one thread per "
                                          "ROI on the caller's records (-1: never)"}
    ctx.close()
    return out


def profile_learned(n, stream):
    """Three learned-start localization calls over n records inside the NVTX
    range "learned" (for ncu --nvtx-include learned/), after training."""
    import torch
    from qcstorm_b200 import lib, synth
    rec, para, _ = synth.gs2d_rois(n, R=R, seed=5)
    net, _ = train_learned_net(para, stream)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = lib.LocContext(para, capacity=n)
    sh = stream.cuda_stream
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("learned")
    for _ in range(3):
        net.localize(ctx, d.data_ptr(), n, 0, iters=LEARNED_ITERS, bisections=LEARNED_BISECTIONS, stream=sh)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile_learned": n, "refits": net.refits(ctx)}))
    ctx.close()
    net.close()
    return 0


def profile_mixed(n, stream):
    """One mixed-size call (qcs_loc_localize_mixed_device) over n records of
    each size of the mixed 7/9/11 workload, then the same records as three
    per-size calls, twice, inside the NVTX range "mixed" (for ncu)."""
    import torch
    from qcstorm_b200 import lib, synth_torch as ST
    data = []
    for i, (kind, R_, _, _) in enumerate(MIXED_SHAPES):
        d, _ = ST.rois(kind, n, R_, seed=30_000 + i, device="cuda")
        data.append((ST.para(kind, R_), d))
    ctxs = [lib.LocContext(p, capacity=n) for p, _ in data]
    ents = [(c, d.data_ptr(), n) for c, (_, d) in zip(ctxs, data)]
    sh = stream.cuda_stream
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("mixed")
    for _ in range(2):
        lib.localize_mixed_device(ents, sh)
        for c, ptr, m in ents:
            c.localize_device(ptr, m, 0, sh)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile_mixed": n}))
    for c in ctxs:
        c.close()
    return 0


def profile_conv(n, stream):
    """The convolutional start-point network's inference (conv_tc_kernel +
    fc_tc_kernel) three times over n GS2D 7x7 records, untrained weights
    (the kernels' work does not depend on the values), for ncu."""
    import torch
    from qcstorm_b200 import lib, synth
    rec, para, _ = synth.gs2d_rois(n, R=R, seed=5)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    net = lib.LearnedNet(batch=1024, seed=4, arch="conv")
    for _ in range(3):
        net.start(para, d.data_ptr(), n, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    net.fused_status()
    print(json.dumps({"profile_conv": n}))
    net.close()
    return 0


def profile_train(n, stream):
    """One training epoch of the MLP and of the conv start-point network over
    n GS2D 7x7 records labelled by plain fits (tcgen05 GEMMs), for ncu."""
    import torch
    from qcstorm_b200 import lib, synth
    rec, para, _ = synth.gs2d_rois(n, R=R, seed=5)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    sh = stream.cuda_stream
    ctx = lib.LocContext(para, capacity=n)
    ctx.localize_device(d.data_ptr(), n, 0, sh)
    feat, scale = lib.LearnedNet.features(para, d.data_ptr(), n, stream=sh)
    tgt, valid = lib.LearnedNet.targets(para, d.data_ptr(), ctx.device_rows(), scale, n, stream=sh)
    out = {}
    for arch in ("mlp", "conv"):
        net = lib.LearnedNet(batch=4096, seed=5, arch=arch)
        out[arch] = float(net.train(feat, tgt, valid, epochs=1, lr=1e-3, stream=sh)[0])
        net.fused_status()
        net.close()
    ctx.close()
    print(json.dumps({"profile_train": n, "loss": out}))
    return 0


def profile_multi(n, stream):
    """The 1-3 emitter 11x11 workload for ncu: networks trained as in
    learned_shapes_measure (count classes, two- and three-emitter starts,
    SHAPE_TRAIN records), then one plain localization call over n records
    inside the NVTX range "plain" and three learned calls (two-emitter starts
    with plain refits of the poor fits, three-emitter starts without refits:
    the fastest variant) inside "learned"."""
    import torch
    from qcstorm_b200 import lib, synth
    Rm = 11
    sh = stream.cuda_stream
    tr, para, _ = synth.multi_rois(SHAPE_TRAIN, R=Rm, seed=7000)
    d_tr = torch.from_numpy(tr.view(np.int16)).cuda()
    ctx_tr = lib.LocContext(para, capacity=SHAPE_TRAIN)
    lib.set_three_emitter_capture(ctx_tr)
    ctx_tr.localize_device(d_tr.data_ptr(), SHAPE_TRAIN, 0, sh)
    labels = lib.count_labels(ctx_tr, SHAPE_TRAIN, sh)
    feat, scale = lib.LearnedNet.features(para, d_tr.data_ptr(), SHAPE_TRAIN, stream=sh)
    tgt, valid = lib.LearnedNet.targets(para, d_tr.data_ptr(), ctx_tr.device_rows(), scale, SHAPE_TRAIN, stream=sh)
    stream.synchronize()
    valid = valid * (labels == 0).float()
    torch.cuda.synchronize()
    net = lib.LearnedNet(batch=4096, seed=5, loc_type=para.LocType, roi_size=Rm)
    net.train(feat, tgt, valid, epochs=TRAIN_EPOCHS, lr=2e-3, stream=sh, classes=labels)
    net.set_count_threshold(0.5)
    net2 = train_two_emitter_net(ctx_tr, para, d_tr, feat, scale, SHAPE_TRAIN, Rm, TRAIN_EPOCHS, stream)
    net.set_two_emitter(net2, iters=TWO_ITERS, bisections=6, fallback="plain")
    net3 = train_three_emitter_net(ctx_tr, para, d_tr, feat, scale, SHAPE_TRAIN, Rm, TRAIN_EPOCHS, stream)
    net.set_three_emitter(net3, iters=THREE_ITERS, bisections=6, dev_th=-1.0)
    ctx_tr.close()
    rec, _, _ = synth.multi_rois(n, R=Rm, seed=8000)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = lib.LocContext(para, capacity=n)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("plain")
    ctx.localize_device(d.data_ptr(), n, 0, sh)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    torch.cuda.nvtx.range_push("learned")
    for _ in range(3):
        net.localize(ctx, d.data_ptr(), n, iters=2, bisections=6, stream=sh)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile_multi": n, "refits": net.refits(ctx)}))
    ctx.close()
    net.set_two_emitter(None)
    net2.close()
    net.set_three_emitter(None)
    net3.close()
    net.close()
    return 0


def profile_fit(n):
    """Three launches of the single-emitter fit kernel over n records."""
    import torch
    from qcstorm_b200 import lib, synth
    rec, para, _ = synth.gs2d_rois(n, R=R, seed=5)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = lib.LocContext(para, capacity=n)
    w = torch.empty((n, 6), dtype=torch.float32, device="cuda")
    sh = torch.cuda.current_stream().cuda_stream
    lib.check(lib.load().qcs_wle_estimate_device(ctx.h, C.c_void_p(d.data_ptr()), n, C.byref(para),
                                                 C.c_void_p(w.data_ptr()), C.c_void_p(sh)))
    out = torch.empty((n, 12), dtype=torch.float32, device="cuda")
    for _ in range(3):
        lib.fit_single_device(0, para, d.data_ptr(), w.data_ptr(), n, out.data_ptr(), sh)
        lib.crlb_device(para, out.data_ptr(), n, sh)
    torch.cuda.synchronize()
    print(json.dumps({"profile_fit": n, "accepted": float((out[:, 0] > 0).float().mean())}))
    ctx.close()
    return 0


def profile_frames(calls, stream):
    """`calls` localization calls of the whole-frame pipeline (for ncu captures)."""
    r = frame_pipeline(stream, steps=calls, warmup=0, e2e=False)
    print(json.dumps({"profile_frames": calls, "frames_per_call": FRAMES_PER_CALL,
                      "records_per_call": r["records_per_call"]}))
    return 0


def free_port():
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def relaunch(n):
    """`bench.py --gpus N` started without a launcher: run it again as N ranks
    (one process per GPU) under torch.distributed.run on this node, bounded by
    `timeout` well above the process group's own timeout."""
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(n), "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-frames", action="store_true", help="skip the whole-frame pipeline measurement")
    ap.add_argument("--profile-fit", type=int, default=0, metavar="N",
                    help="only run the single-emitter fit and CRLB kernels 3 times on N records (for ncu captures)")
    ap.add_argument("--profile-frames", type=int, default=0, metavar="K",
                    help="only run K calls of the whole-frame pipeline (for ncu captures)")
    ap.add_argument("--profile-multi", type=int, default=0, metavar="N",
                    help="trained 1-3 emitter 11x11 networks, then one plain and three learned calls over N records "
                         "in the NVTX ranges plain and learned (for ncu)")
    ap.add_argument("--profile-learned", type=int, default=0, metavar="N",
                    help="only train the start-point network and run 3 learned-start calls on N records")
    ap.add_argument("--profile-conv", type=int, default=0, metavar="N",
                    help="only run the conv start-point network's inference 3 times on N records (for ncu)")
    ap.add_argument("--profile-train", type=int, default=0, metavar="N",
                    help="only run one training epoch of each start-point network on N records (for ncu)")
    ap.add_argument("--profile-mixed", type=int, default=0, metavar="N",
                    help="one mixed-size call and the same records as per-size calls, twice, N records per size "
                         "(for ncu)")
    ap.add_argument("--mixed-persistent", action="store_true",
                    help="only run the plain mixed 7/9/11 measurement (persistent launch against per-size calls)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-start measurement")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed 7/9/11 learned measurement (4e6 training, 1e7 evaluation records)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args.gpus)

    world = env_int("WORLD_SIZE", 1)
    args.gpus = world  # the line reports the ranks that actually ran
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import torch
    from qcstorm_b200 import lib, synth

    torch.cuda.set_device(local)
    # a created stream: the default stream's handle is 0, which the C ABI reads
    # as "the context's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    if args.profile_fit:
        return profile_fit(args.profile_fit)
    if args.profile_frames:
        return profile_frames(args.profile_frames, stream)
    if args.profile_learned:
        return profile_learned(args.profile_learned, stream)
    if args.profile_multi:
        return profile_multi(args.profile_multi, stream)
    if args.profile_conv:
        return profile_conv(args.profile_conv, stream)
    if args.profile_train:
        return profile_train(args.profile_train, stream)
    if args.profile_mixed:
        return profile_mixed(args.profile_mixed, stream)
    if args.mixed_persistent:
        print(json.dumps(mixed_persistent_measure([stream] + [torch.cuda.Stream() for _ in range(IN_FLIGHT - 1)], None,
                                                  1, 0)))
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    # ---- inputs: BATCHES distinct batches resident in HBM, pinned host copies
    d_batches, h_batches = [], []
    para = None
    rec0 = truth0 = None
    for b in range(BATCHES):
        rec, para, truth = synth.gs2d_rois(N_PER_STEP, R=R, seed=batch_seed(rank, b))
        if b == 0:
            rec0, truth0 = rec, truth
        h = torch.from_numpy(rec.view(np.int16)).pin_memory()
        h_batches.append(h)
        d_batches.append(h.cuda())
    ctx = lib.LocContext(para, capacity=N_PER_STEP)
    # IN_FLIGHT contexts in turn, each call on its own stream (the other measurements: two)
    ctxs = [ctx] + [lib.LocContext(para, capacity=N_PER_STEP) for _ in range(IN_FLIGHT - 1)]
    streams = [stream, torch.cuda.Stream()]
    streams_main = streams + [torch.cuda.Stream() for _ in range(IN_FLIGHT - 2)]
    sh = stream.cuda_stream

    def step(k, s, c=None):
        (c or ctxs[k % IN_FLIGHT]).localize_device(d_batches[k % BATCHES].data_ptr(), N_PER_STEP, 0, s.cuda_stream)

    # psf_width, nn_keys_flag, the sort's condition kernel (the sort itself only for out-of-order records),
    # nn_scan_select, classify, init_counters, fit, finish, crlb
    launches_per_step = 9

    # ---- device-timed steps: IN_FLIGHT contexts in turn on their streams
    sampler, spath = start_clock_sampler(local)
    time.sleep(0.5)  # first nvidia-smi sample lands before the timed region
    t_start = time.time()
    ms, windows = device_timed_windows(args.steps, args.warmup, step, streams_main, dist)
    t_end = time.time()
    clocks = stop_clock_sampler(sampler, spath, t_start, t_end)
    value = job_rate(args.steps, N_PER_STEP, world, ms)
    one_steps = min(args.steps, 200)
    ms1 = device_timed(one_steps, 3, lambda k, s: step(k, s, ctx), [stream], dist)
    value1 = job_rate(one_steps, N_PER_STEP, world, ms1)

    # ---- dominant kernel alone: the single-emitter fit (for the roofline)
    wle_b = [torch.empty((N_PER_STEP, 6), dtype=torch.float32, device="cuda") for _ in range(BATCHES)]
    for b in range(BATCHES):
        lib.load().qcs_wle_estimate_device(ctx.h, C.c_void_p(d_batches[b].data_ptr()), N_PER_STEP, C.byref(para),
                                           C.c_void_p(wle_b[b].data_ptr()), C.c_void_p(sh))
    d_loc = torch.empty((N_PER_STEP, 12), dtype=torch.float32, device="cuda")
    for k in range(3):
        lib.fit_single_device(0, para, d_batches[k].data_ptr(), wle_b[k].data_ptr(), N_PER_STEP, d_loc.data_ptr(), sh)
    torch.cuda.synchronize()
    kt = []
    for k in range(min(args.steps, 50)):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        lib.fit_single_device(0, para, d_batches[k % BATCHES].data_ptr(), wle_b[k % BATCHES].data_ptr(), N_PER_STEP,
                              d_loc.data_ptr(), sh)
        b.record(stream)
        kt.append((a, b))
    torch.cuda.synchronize()
    fit_ms = statistics.mean(a.elapsed_time(b) for a, b in kt)
    mufu_peak = lib.mufu_rate()
    achieved = N_PER_STEP * PX_EVALS_PER_FIT * MUFU_PER_PX_EVAL / (fit_ms * 1e-3)

    # ---- end to end through the host-buffer calls (pinned records in, rows out every step)
    e2e_pipelined(ctxs, streams_main, h_batches, 4)
    e2e_steps = E2E_STEPS
    e2e_s, rows = e2e_pipelined(ctxs, streams_main, h_batches, e2e_steps)
    e2e_s = max_over_ranks(e2e_s * 1e3, dist) * 1e-3
    # the synchronous reference-shaped call, one at a time
    sync_steps = 10
    for k in range(2):
        ctx.localize(h_batches[k].numpy().view(np.uint16), None, stream=sh, copy=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(sync_steps):
        ctx.localize(h_batches[k % BATCHES].numpy().view(np.uint16), None, stream=sh, copy=False)
    sync_s = max_over_ranks((time.perf_counter() - t0) * 1e3, dist) * 1e-3
    e2e = {"value": e2e_steps * N_PER_STEP * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": N_PER_STEP * R * (R + 1) * 2,
           "d2h_bytes_per_step": int(rows / e2e_steps) * 48 + 32,
           "call": "qcs_loc_localize_async + qcs_loc_finish on three contexts in turn (pinned host records in, rows "
                   "and counters out every step, WLE on device)",
           "sync_value": sync_steps * N_PER_STEP * world / sync_s,
           "sync_call": "qcs_loc_bfgs_mle_localization, one call at a time (rows read in place from h_LocArry)"}

    learned = None
    if not args.no_learned:
        learned = learned_measure(args, streams_main, ctxs, para, d_batches, h_batches, rec0, truth0, value, world,
                                  dist)

    consec = consec_measure(stream, dist, world)
    tune = autotune_measure(stream, dist, world)

    shapes = mixed = None
    if not args.no_learned:
        shapes = learned_shapes_measure(streams_main, dist, world, rank, mufu_peak=mufu_peak,
                                        cpu_baseline=not args.no_cpu_baseline)
        if not args.no_mixed:
            mixed = mixed_measure(streams_main, dist, world, rank)
            mixed["plain_persistent"] = mixed_persistent_measure(streams_main, dist, world, rank)

    frames = None
    if not args.no_frames:
        fsteps = min(max(args.steps // 40, 5), 40)
        frames = frame_pipeline(stream, steps=fsteps, warmup=3, dist=dist, world=world)
        st = frames["stages"]
        ops = cascade_mufu_ops(R, st["single"], st["two_emitter"], st["three_emitter"])
        frames["roofline"] = {
            "bound": "sfu", "unit": "MUFU op/s", "peak": mufu_peak,
            "achieved": ops / (frames["ms_per_call"] * 1e-3), "frac": ops / (frames["ms_per_call"] * 1e-3) / mufu_peak,
            "scope": "whole call (32 extractions + localization cascade + CRLB); fits counted on the reference "
                     "schedule; frames read once from HBM: %.1f GB/s" % (
                         FRAMES_PER_CALL * FRAME_W * FRAME_H * 2 / (frames["ms_per_call"] * 1e-3) / 1e9)}
        if rank == 0 and not args.no_cpu_baseline:
            frames["cpu_baseline"] = frame_cpu_baseline()
        if not args.no_learned:
            frames["learned"] = frame_pipeline_learned(stream, fsteps, 3, dist=dist, world=world)
            frames["learned"]["vs_plain"] = frames["learned"]["frames_per_s"] / frames["frames_per_s"]
            frames["learned_multi_starts"] = frame_pipeline_learned(stream, fsteps, 3, dist=dist, world=world,
                                                                    multi_starts=True)
            frames["learned_multi_starts"]["vs_plain"] = (frames["learned_multi_starts"]["frames_per_s"] /
                                                          frames["frames_per_s"])

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu, _ = cpu_reference_rate(steps=1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_dict(args),
            "windows": windows, "window_note": "value = median over %d device-timed windows of exactly %d steps "
                                              "(repeated to >= %.0f ms so the clock samples cover them)" % (
                                                  windows, args.steps, MIN_TIMED_MS),
            "value_one_stream": value1, "timing": "three contexts in turn on three streams, CUDA events around all "
                                                  "(value_one_stream: one context, one stream)",
            "e2e": e2e, "gpu_launches": launches_per_step * args.steps * windows,
            "roofline": {"bound": "sfu", "kernel": "fit_single_kernel<7,GS2D>", "achieved": achieved,
                         "peak": mufu_peak, "unit": "MUFU op/s", "frac": achieved / mufu_peak,
                         "traffic": DRAM_BYTES_PER_FIT * N_PER_STEP,
                         "traffic_algorithmic": ALGO_BYTES_PER_FIT * N_PER_STEP,
                         "traffic_note": "DRAM bytes per launch from ncu on 200 k records, scaled to %d" % N_PER_STEP,
                         "kernel_ms": fit_ms,
                         "algorithmic": "%d px-evals x %d MUFU per fit; peak = measured __expf/__logf rate" % (
                             PX_EVALS_PER_FIT, MUFU_PER_PX_EVAL)},
            "cpu_baseline": cpu, "clocks": clocks, "learned": learned, "learned_other_configs": shapes,
            "learned_mixed_7_9_11": mixed,
            "consecutive_fit": consec, "autotune": tune,
            "frames": frames,
        }
        if learned:
            a = learned["accuracy"]
            line.update({
                "learned_value": learned["value"], "learned_vs_plain": learned["vs_plain"],
                "learned_e2e_value": learned["e2e"]["value"],
                "learned_rmse_px": a["rmse_px"]["learned"], "plain_rmse_px": a["rmse_px"]["plain"],
                "learned_rmse_px_own": a["own_accepted"]["rmse_px"]["learned"],
                "plain_rmse_px_own": a["own_accepted"]["rmse_px"]["plain"],
                "learned_accept": a["accepted"]["learned"], "plain_accept": a["accepted"]["plain"],
                "learned_equal_rmse": a["equal_rmse"], "crlb_px": a["crlb_px"],
                "fisher_crlb_px": a["fisher_crlb"]["plain"]["crlb_px"],
                "plain_rmse_over_fisher_crlb": a["fisher_crlb"]["plain"]["rms_error_over_own_crlb"],
                "learned_rmse_over_fisher_crlb": a["fisher_crlb"]["learned"]["rms_error_over_own_crlb"],
                "learned_equal_rmse_within_2pct_of_crlb": a["fisher_crlb"]["equal_rmse_within_2pct_of_crlb"],
                "learned_no_refit_value": learned["no_refit"]["value"],
                "learned_no_refit_vs_plain": learned["no_refit"]["vs_plain"],
                "learned_no_refit_rmse_px": learned["no_refit"]["rmse_px"]["no_refit"],
                "learned_no_refit_accept": learned["no_refit"]["accepted"],
                "learned_conv_value": learned["conv"]["value"], "learned_conv_vs_plain": learned["conv"]["vs_plain"],
                "learned_conv_rmse_px": learned["conv"]["accuracy"]["rmse_px"]["conv"],
            })
        # short keys first: the headline survives a truncated tail of the line
        head = ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "learned_value", "learned_vs_plain", "learned_e2e_value",
                "learned_rmse_px", "plain_rmse_px", "learned_rmse_px_own", "plain_rmse_px_own", "learned_accept",
                "plain_accept", "learned_equal_rmse", "crlb_px", "fisher_crlb_px", "plain_rmse_over_fisher_crlb",
                "learned_rmse_over_fisher_crlb", "learned_equal_rmse_within_2pct_of_crlb", "learned_no_refit_value",
                "learned_no_refit_vs_plain", "learned_no_refit_rmse_px", "learned_no_refit_accept", "learned_conv_value",
                "learned_conv_vs_plain", "learned_conv_rmse_px", "gpu_launches", "windows",
                "clocks", "roofline",
                "e2e", "cpu_baseline", "config"]
        line = {**{k: line[k] for k in head if k in line}, **{k: v for k, v in line.items() if k not in head}}
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
