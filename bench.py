"""Benchmark of the BAM reader hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config gex|small|atac|uneven|serve|bai|write]

One step = one decode of the whole synthetic BAM of the workload (default: the
GEX-shaped batch, 50,000,000 single-end 91 bp records over the 25 human
chromosomes): BGZF member scan, inflate with CRC32/ISIZE checks, record chain,
fixed columns and the CB/UB/GN tags.  The metric is GB/s of decompressed
(uncompressed) BAM bytes, whole job over all ranks; records/s rides along.

- ``value``: the batched decoder (``cubam_b200.batch``) with the compressed file
  resident in HBM (one persistent inflate launch for all members), timed with
  CUDA events between barriers, max over ranks.  Inputs (4-5 GB compressed,
  12.6 GB inflated) are far larger than the 126 MB L2, so no flush is needed.
- ``e2e``: the public API, ``cubam_b200.read_bam(path)`` from the page cache with
  the CB/UB/GN tags decoded per batch: pread into pinned buffers, H2D copies, all
  kernels, and a D2H read of the per-step checksum, timed by the device clock.
- ``roofline``: the inflate kernel (the dominant one): decompressed bytes per
  launch / its CUDA-event duration, against the measured HBM copy bandwidth.
- ``serving``: the serving loop on the same file, bounded (100 requests of log-uniform
  64 KB-512 MB compressed ranges, all at once, then Poisson at 80% of that rate):
  p50/p95/p99 latency and throughput against the batched decode.
- ``cpu_baseline``: the C oracle (zlib inflate + record chain + columns, all host
  cores) on a bounded prefix of the same file; ``parity`` compares the GPU's
  records, columns and tags of that prefix with the oracle's ("ok" or the first
  mismatch).
- ``--impl reference``: cubam's reader needs CuPy, cuDF and nvCOMP and has no
  CPU path; the reference arm times the CPU restatement of its reader path
  (``oracle/cpu_decoder.c``, all host cores) on the whole file of the same
  workload per step, rank 0 only.  That process loads nothing of ``cubam_b200``:
  the input file is written by the generator's executable in a child process.

Multi-GPU (torchrun): every rank decodes its own copy of the file (replicas: the
path shards by file with no exchange), ``scaling`` = weak.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "BAM decode GB/s (uncompressed) & records/s on 1 B200"
UNIT = "GB/s"
FALLBACK_HBM = 6650.0
#: DRAM bytes (read + write) per inflated byte of each inflate form, from one ncu capture each on the
#: 4M-record GEX file (1,008,824,685 inflated bytes); the bench scales them by its inflated bytes
TRAFFIC_PER_BYTE = {"k_inflate_lanes": (6.916637e9 + 1.003612e9) / 1.008824685e9,
                    "k_inflate_warp": (1.593613e9 + 1.004537e9) / 1.008824685e9,
                    "k_decode + k_copy": (0.414233344e9 + 0.754765312e9 + 1.45392e9 + 0.958392832e9) / 1.008824685e9}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="gex", choices=["gex", "small", "atac", "uneven", "serve", "bai", "write"])
    ap.add_argument("--level", type=int, default=2, help="write: DEFLATE level")
    ap.add_argument("--write-gb", type=float, default=1.0, help="write: input GB (tiled copies of the synthetic file)")
    ap.add_argument("--rate", type=float, default=0.0,
                    help="serve: Poisson arrivals per second (0: the rate that offers 80%% of the saturation throughput)")
    ap.add_argument("--requests", type=int, default=400, help="serve: requests")
    ap.add_argument("--file-records", type=int, default=4_000_000, help="serve: records per resident file")
    ap.add_argument("--scale", type=float, default=1.0, help="uneven: record counts times this")
    ap.add_argument("--records", type=int, default=None, help="override the workload size (records)")
    ap.add_argument("--chunk-bytes", type=int, default=None,
                    help="compressed chunk of the e2e read_bam (default: read_bam's own, auto_chunk_bytes())")
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--cpu-sample-mb", type=int, default=2048, help="compressed MB of the CPU baseline sample")
    ap.add_argument("--workdir", default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="gex: skip the bounded serving sub-object")
    ap.add_argument("--form", type=int, default=0,
                    help="inflate form for every batch size (1 warp per member, 2 lane per member, 3 split); "
                         "0: the library's choice")
    return ap.parse_args()


def max_over_ranks(ms: float) -> float:
    """The largest of the ranks' times (every rank gets it): NCCL on the GPU, gloo on the host."""
    import torch
    import torch.distributed as td

    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return ms
    dev = "cuda" if td.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def whole_job(units_per_rank: float, ms: float, world: int) -> float:
    """Weak scaling: every rank processed the same units; the job's rate over the slowest rank's time."""
    return units_per_rank * world / (ms / 1e3)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM)), "measured"
    return FALLBACK_HBM, "fallback"


def _synth():
    """``cubam_b200/synth.py`` loaded on its own: the generator's configurations without importing the
    package (whose import loads the decoder's library)."""
    import importlib.util

    mod = sys.modules.get("_cubam_synth")
    if mod is None:
        spec = importlib.util.spec_from_file_location("_cubam_synth", ROOT / "cubam_b200" / "synth.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules["_cubam_synth"] = mod
        spec.loader.exec_module(mod)
    return mod


def workload(args):
    synth = _synth()
    cfg = synth.CONFIGS[args.config]
    n = args.records or cfg.n_records
    base = Path(args.workdir or ("/dev/shm" if Path("/dev/shm").exists() else "/tmp"))
    path = base / f"cubam_bench_{cfg.name}_{n}_s{cfg.seed}.bam"
    return cfg, n, path


def ensure_file(args, rank, dist):
    cfg, n, path = workload(args)
    t = 0.0
    if rank == 0 and not path.exists():
        t0 = time.perf_counter()
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        _synth().write_bam_process(tmp, cfg, n_records=n)
        tmp.replace(path)
        t = time.perf_counter() - t0
    if dist:
        import torch.distributed as td

        td.barrier()
    return cfg, n, path, t


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200", "-i",
                 str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(path: Path, sample_mb: int):
    """The C oracle on the first ``sample_mb`` MB of compressed members, all host cores: the baseline
    figure and the decoded sample (the checker of the GPU's records)."""
    import numpy as np

    from oracle import cpu_oracle

    raw = np.fromfile(path, dtype=np.uint8)
    cores = os.cpu_count() or 1
    ws = {}
    cpu_oracle.decode_prefix(raw, sample_mb << 20, cores, ws=ws)  # warm-up: page faults of fresh buffers
    secs, d = None, None
    for _ in range(2):
        d = cpu_oracle.decode_prefix(raw, sample_mb << 20, cores, ws=ws)
        secs = d.seconds["total"] if secs is None else min(secs, d.seconds["total"])
    return d, {
        "value": d.inflated_bytes / secs / 1e9,
        "unit": UNIT,
        "cores": cores,
        "kind": "port",
        "sample": f"first {d.n_members} members ({d.compressed_bytes / 1e6:.0f} MB compressed, "
                  f"{d.inflated_bytes / 1e6:.0f} MB inflated, {len(d.offset)} records) of the same file: zlib "
                  f"inflate + record chain + columns + CB/UB/GN tags in {secs:.2f} s",
        "records_per_s": len(d.offset) / secs,
    }


def run_reference(args):
    """CPU restatement of the reference's reader path (the reference has no CPU path of its own): every
    step decodes the whole file of the workload (all members, records, columns and CB/UB/GN tags) on all
    host cores.  Nothing of ``cubam_b200`` is imported or loaded in this process."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, n, path, gen_s = ensure_file(args, 0, None)
    import numpy as np

    from oracle import cpu_oracle

    raw = np.fromfile(path, dtype=np.uint8)
    cores = os.cpu_count() or 1
    ws = {}  # output arrays kept between steps, so steps do not fault in fresh pages
    for _ in range(args.warmup):
        cpu_oracle.decode_file(raw, cores, ws=ws)
    times, inflated, recs, members = [], 0, 0, 0
    for _ in range(args.steps):
        d = cpu_oracle.decode_file(raw, cores, ws=ws)
        times.append(d.seconds["total"])
        inflated, recs, members = d.inflated_bytes, len(d.offset), d.n_members
    ms = statistics.mean(times) * 1e3
    value = inflated / (ms / 1e3) / 1e9
    sample = (f"the whole file per step: {members} members ({raw.size / 1e6:.0f} MB compressed, "
              f"{inflated / 1e6:.0f} MB of records inflated, {recs} records), zlib inflate + record chain + "
              f"columns + CB/UB/GN tags")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"{cfg.name}: {n} records, zlib level {cfg.level}, seed {cfg.seed}",
                   "records_per_step": recs, "generate_s": round(gen_s, 1)},
        "records_per_s": recs / (ms / 1e3),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def parity(gpu, ref, tags) -> str:
    """"ok" when the GPU's decode of a file starts with the oracle's records (offsets, the 11 fixed columns,
    and type/offset/length/value of each tag), else the first mismatch."""
    import numpy as np

    from cubam_b200.bam import FIELDS

    n = len(ref.offset)
    if len(gpu) < n:
        return f"records: {len(gpu)} on the GPU, {n} in the oracle's sample"

    def first_diff(name, a, b):
        bad = np.flatnonzero(a != b)
        return f"{name}: record {int(bad[0])}: GPU {a[bad[0]]}, oracle {b[bad[0]]}" if bad.size else None

    checks = [("offset", gpu.offset[:n], ref.offset)]
    checks += [(f, gpu.columns[f][:n], ref.columns[f]) for f in FIELDS]
    for t in tags:
        g = gpu.tags[t]
        ty, vo, vl, iv, _ = ref.tags[t]
        checks += [(f"{t}.type", g.type[:n], ty), (f"{t}.offset", g.offset[:n], vo), (f"{t}.length", g.length[:n], vl),
                   (f"{t}.value", g.value[:n], iv)]
    for name, a, b in checks:
        msg = first_diff(name, a.cpu().numpy(), np.asarray(b))
        if msg:
            return msg
    return "ok"


def run_ours(args):
    import torch

    dist = int(os.environ.get("WORLD_SIZE", "1")) > 1
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    if dist:
        import datetime

        import torch.distributed as td

        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    cfg, n, path, gen_s = ensure_file(args, rank, dist)

    import cubam_b200
    from cubam_b200 import _lib, batch

    if args.form:
        _lib.lib.cb_set_param(_lib.PARAM_INFLATE_FORM, args.form)
        _lib.lib.cb_set_param(_lib.PARAM_SPLIT_MIN_JOBS, 0)

    header = cubam_b200.BamHeader.read(path)
    comp = batch.load_compressed(path)
    torch.cuda.synchronize()
    counter = {}
    tags = ("CB", "UB", "GN")

    def step(ev=None, cnt=None):
        return batch.decode_resident(comp, header, tags=tags, events=ev, counter=cnt)

    for _ in range(max(args.warmup, 0)):
        res = step()
        del res
    torch.cuda.synchronize()
    res = step()
    inflated = res.inflated_bytes
    n_rec = len(res)
    n_members = res.n_members
    del res

    def barrier():
        if dist:
            import torch.distributed as td

            td.barrier()

    evs = []
    with Clocks(local) as clk:
        barrier()
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(args.steps):
            ev = batch.StageEvents()
            r = step(ev, counter)
            evs.append(ev)
            del r
        stop.record()
        torch.cuda.synchronize()
        barrier()
    ms = start.elapsed_time(stop) / args.steps
    if dist:
        ms = max_over_ranks(ms)
    stage = {k: statistics.mean(e.ms()[k] for e in evs) for k in evs[0].ms()}
    inflate_ms = stage["inflated"]
    value = whole_job(inflated, ms, world) / 1e9
    peak, peak_kind = peaks()
    achieved = inflated / (inflate_ms / 1e3) / 1e9
    from cubam_b200.bgzf import inflate_form

    form = inflate_form(0, n_members)  # the form the batched decode runs
    kernel = {1: "k_inflate_warp", 2: "k_inflate_lanes", 3: "k_decode + k_copy"}[form]

    # the plain per-chunk form of the same kernels on device-resident chunks (cubam's structure)
    plain = None
    if not args.no_plain:
        plain = plain_per_chunk(comp, header, args.chunk_bytes or (256 << 20), tags)

    fused = fused_record_pass(comp, header) if rank == 0 else None
    serving = serving_probe(path, value / world, tags) if rank == 0 and not args.no_serving else None

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(path, args, tags, inflated, rank, dist)
    cpu, checked = None, None
    if rank == 0 and not args.no_cpu:
        ref, cpu = cpu_baseline(path, args.cpu_sample_mb)
        res = step()  # one more decode of the whole file, its records checked against the oracle's sample
        checked = {"result": parity(res, ref, tags), "records": len(ref.offset), "of": n_rec,
                   "compared": "offsets, 11 fixed columns, CB/UB/GN type/offset/length/value"}
        del res, ref
    if rank != 0:
        if dist:
            import torch.distributed as td

            td.destroy_process_group()
        return
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": {
            "workload": f"{cfg.name}: {n} records, zlib level {cfg.level}, seed {cfg.seed}",
            "compressed_bytes": int(comp.numel()),
            "inflated_bytes": inflated,
            "members": n_members,
            "records": n_rec,
            "tags": list(tags),
            "form": "batched: whole file resident, one persistent inflate launch",
            "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"replicas x{world}",
            "generate_s": round(gen_s, 1),
        },
        "records_per_s": n_rec * world / (ms / 1e3),
        "stages_ms": {k: round(v, 3) for k, v in stage.items()},
        "roofline": {
            "bound": "hbm",
            "kernel": kernel,
            "form": form,
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "peak_kind": peak_kind,
            "algorithmic": "decompressed bytes (sum of ISIZE) per launch",
            # DRAM bytes (read + write) per inflated byte of the kernel, measured by ncu on the
            # 4M-record GEX case, scaled by the launch's inflated bytes
            "traffic": inflated * TRAFFIC_PER_BYTE[kernel] if kernel in TRAFFIC_PER_BYTE else None,
        },
        "clocks": clk.summary(),
        "gpu_launches": counter.get("launches", 0),
    }
    if plain:
        line["plain_per_chunk"] = plain
    if fused:
        line["fused_record_pass"] = fused
    if serving:
        line["serving"] = serving
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    if checked:
        line["parity"] = checked
    print(json.dumps(line), flush=True)
    if dist:
        import torch.distributed as td

        td.destroy_process_group()


def serving_probe(path, batch_gbs: float, tags, n_requests: int = 100) -> dict:
    """The serving loop on the bench file, bounded: the file resident once, 100 requests of log-uniform
    64 KB-512 MB compressed ranges (seed 5), first all at once (the loop's saturation throughput),
    then as a Poisson stream at 80% of it; latency percentiles (all requests, and those of at most
    8 MB compressed) and throughput against the batched decode of the whole file."""
    import torch

    from cubam_b200 import serve

    rf = serve.ResidentFile.load(path)
    files = [rf]
    server = serve.Server(files, budget_bytes=40 << 30, tags=tags)

    def sink(r):
        if r.result is not None and len(r.result):
            r.result.columns["pos"].sum()

    server.run(serve.poisson_requests(files, 8, 1e9, seed=6), on_done=sink)  # set every kernel up
    torch.cuda.synchronize()

    def served(rate):
        reqs = serve.poisson_requests(files, n_requests, rate, seed=5)
        t = time.perf_counter()
        done = server.run(reqs, on_done=sink, t0=t)
        torch.cuda.synchronize()
        span = time.perf_counter() - t
        return {"throughput_gbs": sum(r.inflated_bytes for r in done) / span / 1e9, "span_s": round(span, 4),
                **serve.latency_summary(done)}, done

    sat, done = served(1e9)
    mean = sum(r.inflated_bytes for r in done) / len(done)
    rate = 0.8 * sat["throughput_gbs"] * 1e9 / mean
    live, done = served(rate)
    out = {"requests": n_requests, "files": 1, "rate_per_s": round(rate, 2),
           "sizes": "log-uniform 64 KB-512 MB compressed ranges of the bench file, seed 5",
           "small": "at most 8 MB compressed", "saturation": sat, "served": live,
           "served_vs_batch": live["throughput_gbs"] / batch_gbs,
           "saturation_vs_batch": sat["throughput_gbs"] / batch_gbs,
           "batch_gbs": batch_gbs}
    del server, files, rf
    torch.cuda.empty_cache()
    return out


def fused_record_pass(comp, header):
    """Columns + aligned length + read-name hash of all records: three kernels (fixed columns, then the two
    on-request decoders, each reading the records again) against one fused pass (cb_decode_records)."""
    import torch

    from cubam_b200 import _lib, batch
    from cubam_b200.bam import _TYPES, FIELDS
    from cubam_b200.bgzf import stream_ptr

    d = batch.decode_resident(comp, header, tags=())
    n = len(d)
    cols = {k: torch.empty(n, dtype=t, device="cuda") for k, t in _TYPES.items()}
    al = torch.empty(n, dtype=torch.int32, device="cuda")
    nh = torch.empty(n, dtype=torch.uint64, device="cuda")
    ptrs = [cols[k].data_ptr() for k in FIELDS]
    data, off, s = d.data.data_ptr(), d.offset.data_ptr(), stream_ptr()

    def separate():
        _lib.lib.cb_decode_fixed(data, off, n, *ptrs, s)
        _lib.lib.cb_aligned_length(data, off, n, al.data_ptr(), s)
        _lib.lib.cb_name_hash(data, off, n, nh.data_ptr(), s)

    def fused():
        _lib.lib.cb_decode_records(data, off, n, *ptrs, al.data_ptr(), nh.data_ptr(), s)

    out = {"records": n}
    for name, fn in (("separate_ms", separate), ("fused_ms", fused)):
        fn()
        times = []
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        out[name] = min(times)
    del d
    return out


def plain_per_chunk(comp, header, chunk_bytes, tags):
    """One pass of the per-chunk form (scan, sync, inflate, chain, sync, decode per chunk) on resident chunks."""
    import torch

    from cubam_b200 import _lib
    from cubam_b200.bam import RecordBatch, record_chain
    from cubam_b200.bgzf import _inflate_blocks, check_inflate, raise_status, read_struct

    def one_pass():
        n = int(comp.numel())
        carry_c = torch.empty(0, dtype=torch.uint8, device="cuda")
        carry_r = torch.empty(0, dtype=torch.uint8, device="cuda")
        skip = header.size
        recs = 0
        for a in range(0, n, chunk_bytes):
            b = min(a + chunk_bytes, n)
            buf = torch.cat([carry_c, comp[a:b]]) if carry_c.numel() else comp[a:b]
            data, used, summ = _inflate_blocks(buf, b >= n, carry_r, True, True)
            carry_c = buf[used:].clone()
            if skip:
                k = min(skip, int(data.numel()))
                data = data[k:]
                skip -= k
            if int(data.numel()) == 0:
                carry_r = data
                continue
            offsets, cs = record_chain(data, len(header.names))
            if summ is not None:
                check_inflate(summ)
            s = read_struct(cs, _lib.ChainSummary)
            raise_status(s.status, "record chain")
            off = offsets[: s.n_records]
            carry_r = data[s.tail:].clone()
            if off.numel():
                bt = RecordBatch.decode(data, off, header)
                bt.tags(*tags)
                recs += len(bt)
        return recs

    one_pass()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    recs = one_pass()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e)
    return {"ms_per_step": ms, "records": recs, "chunk_bytes": chunk_bytes}


def run_e2e(path, args, tags, inflated, rank, dist):
    """read_bam through the public API, file -> pinned -> device, with a D2H checksum per step."""
    import torch

    import cubam_b200

    size = os.path.getsize(path)
    from cubam_b200 import auto_chunk_bytes

    chunk = args.chunk_bytes or auto_chunk_bytes()

    def one():
        chk = torch.zeros(1, dtype=torch.int64, device="cuda")
        recs = 0
        for b in cubam_b200.read_bam(path, chunk_bytes=chunk):
            for t in b.tags(*tags):
                chk += t.length.sum()
            chk += b.pos.sum()
            recs += len(b)
        return recs, int(chk.item())  # the D2H read of the step's result

    one()
    torch.cuda.synchronize()
    if dist:
        import torch.distributed as td

        td.barrier()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    s.record()
    for _ in range(args.e2e_steps):
        recs, _ = one()
    e.record()
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / args.e2e_steps
    ms = s.elapsed_time(e) / args.e2e_steps
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if dist:
        ms = max_over_ranks(ms)
    return {
        "value": inflated * world / (ms / 1e3) / 1e9,
        "unit": UNIT,
        "h2d_bytes_per_step": size,
        "d2h_bytes_per_step": 8,
        "ms_per_step": ms,
        "wall_ms_per_step": wall * 1e3,
        "records_per_s": recs * world / (ms / 1e3),
        "chunk_bytes": chunk,
        "api": "cubam_b200.read_bam(path) + RecordBatch.tags('CB','UB','GN')",
    }


def run_uneven(args):
    """The uneven-size batch: 64 files (log-uniform 10k-20M records times --scale, GEX or ATAC records,
    zlib levels 1-9 per member, 2% stored members) decoded as one graph-replayed batch (one inflate
    launch for all members, the inflate form chosen by the autotuner) against one decode per file."""
    import torch

    import cubam_b200
    from cubam_b200 import batch, synth

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    base = Path(args.workdir or ("/dev/shm" if Path("/dev/shm").exists() else "/tmp"))
    cfgs = synth.uneven_files(scale=args.scale)
    t0 = time.perf_counter()
    paths = []
    for cfg in cfgs:
        path = base / f"cubam_bench_{cfg.name}_{cfg.n_records}_s{cfg.seed}.bam"
        if not path.exists():
            tmp = path.with_suffix(f".tmp{os.getpid()}")
            synth.write_bam(tmp, cfg)
            tmp.replace(path)
        paths.append(path)
    gen_s = time.perf_counter() - t0
    files = [(batch.load_compressed(p), cubam_b200.BamHeader.read(p)) for p in paths]
    torch.cuda.synchronize()
    plan = batch.BatchPlan(files)
    plan.capture()
    for _ in range(max(args.warmup, 0)):
        plan.replay()
    torch.cuda.synchronize()
    plan.check()
    inflated = sum(plan.inflated)
    n_rec = sum(plan.n_records)
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(args.steps):
            plan.replay()
        e.record()
        torch.cuda.synchronize()
    plan.check()
    ms = s.elapsed_time(e) / args.steps
    ev = batch.StageEvents()
    plan.launch(events=ev)
    torch.cuda.synchronize()
    stage = ev.ms()
    # one decode per file: its own scan, inflate launch, chain and columns, with the host syncs
    for f in files:
        batch.decode_many([f])
    torch.cuda.synchronize()
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record()
    for f in files:
        r = batch.decode_many([f])
        del r
    e2.record()
    torch.cuda.synchronize()
    ms_per_file = s2.elapsed_time(e2)
    peak, peak_kind = peaks()
    achieved = inflated / (stage["inflated"] / 1e3) / 1e9
    kernel = {1: "k_inflate_warp", 2: "k_inflate_lanes", 3: "k_decode + k_copy"}[plan.form]
    print(json.dumps({
        "metric": METRIC, "value": inflated / (ms / 1e3) / 1e9, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"uneven: 64 files, {n_rec} records (log-uniform 10k-20M x {args.scale}), GEX/ATAC, "
                               f"levels 1-9 per member, 2% stored, seed 3",
                   "compressed_bytes": sum(int(c.numel()) for c, _ in files), "inflated_bytes": inflated,
                   "members": sum(plan.n_members), "records": n_rec,
                   "form": "one CUDA graph per step: all scans, ONE inflate launch, all chains and columns",
                   "l2": "inputs larger than L2 (no flush)", "generate_s": round(gen_s, 1)},
        "records_per_s": n_rec / (ms / 1e3),
        "autotune": {"params": plan.tuning["params"], "ms": plan.tuning["ms"], "seconds": plan.tuning["seconds"],
                     "key": plan.tuning["key"]},
        "inflate_form": plan.form,
        "stages_ms": {k: round(v, 3) for k, v in stage.items()},
        "one_launch_per_file": {"ms_per_step": ms_per_file, "value": inflated / (ms_per_file / 1e3) / 1e9,
                                "records_per_s": n_rec / (ms_per_file / 1e3)},
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic": "decompressed bytes (sum of ISIZE) per launch",
                     "traffic": inflated * TRAFFIC_PER_BYTE[kernel] if kernel in TRAFFIC_PER_BYTE else None},
        "clocks": clk.summary(),
        "gpu_launches": plan.launches_per_run(),
    }), flush=True)


def run_serve(args):
    """The serving loop: 16 resident files (GEX and ATAC shapes), requests of log-uniform 64 KB-512 MB
    compressed ranges arriving as a Poisson stream, admitted under a 40 GB HBM budget; latency
    percentiles and throughput of continuous batching against the plain sequential decode (one
    request at a time, in arrival order), and the saturation throughput (all requests at once)."""
    import torch

    from cubam_b200 import serve, synth
    from cubam_b200.synth import Config

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    base = Path(args.workdir or ("/dev/shm" if Path("/dev/shm").exists() else "/tmp"))
    t0 = time.perf_counter()
    files = []
    for i in range(16):
        shape = 1 if i % 2 == 0 else 2
        cfg = Config(f"serve{i}", shape, args.file_records, 4000 + i, n_barcodes=1000 if shape == 1 else 10_000)
        path = base / f"cubam_bench_{cfg.name}_{cfg.n_records}_s{cfg.seed}.bam"
        if not path.exists():
            tmp = path.with_suffix(f".tmp{os.getpid()}")
            synth.write_bam(tmp, cfg)
            tmp.replace(path)
        files.append(serve.ResidentFile.load(path))
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    tags = ("CB", "UB", "GN")
    budget = 40 << 30

    def requests(rate):
        return serve.poisson_requests(files, args.requests, rate, seed=4)

    def sink(r):  # consume the result on the device, as a caller would, then release it
        if r.result is not None and len(r.result):
            r.result.columns["pos"].sum()

    server = serve.Server(files, budget_bytes=budget, tags=tags)
    warm = requests(1e9)[:16]
    server.run(warm, on_done=sink)  # set every kernel up
    torch.cuda.synchronize()

    def served(rate):
        reqs = requests(rate)
        steps0, gpu0, host0 = server.steps, server.gpu_ms, dict(server.host_s)
        with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
            t = time.perf_counter()
            done = server.run(reqs, on_done=sink, t0=t)
            torch.cuda.synchronize()
            span = time.perf_counter() - t
        inflated = sum(r.inflated_bytes for r in done)
        return {"throughput_gbs": inflated / span / 1e9, "span_s": span, "steps": server.steps - steps0,
                "gpu_step_ms": server.gpu_ms - gpu0,
                "host_s": {k: round(v - host0[k], 4) for k, v in server.host_s.items()},
                **serve.latency_summary(done)}, clk.summary(), done

    sat, _, _ = served(1e9)  # every request at once: the loop's batch throughput
    probe = requests(1.0)
    for r in probe:
        serve.plan_request(files[r.file], r)
    mean_bytes = sum(r.inflated_bytes for r in probe) / len(probe)
    rate = args.rate or 0.8 * sat["throughput_gbs"] * 1e9 / mean_bytes
    live, clocks, done = served(rate)
    n_small = sum(1 for r in done if r.compressed_bytes <= (8 << 20))

    # the plain sequential decode: one request at a time in arrival order, each alone
    reqs = requests(rate)
    t = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t
        if r.arrival > now:
            time.sleep(r.arrival - now)
        res = serve.decode_alone(files[r.file], r, tags=tags)
        sink(serve.Request(0, 0, 0, result=res))
        torch.cuda.synchronize()
        r.done = time.perf_counter() - t
        del res
    span = time.perf_counter() - t
    plain = {"throughput_gbs": sum(r.inflated_bytes for r in reqs) / span / 1e9, "span_s": span,
             **serve.latency_summary(reqs)}
    total = sum(r.inflated_bytes for r in done)
    print(json.dumps({
        "metric": METRIC, "value": live["throughput_gbs"], "unit": UNIT, "n_gpus": 1, "steps": args.requests,
        "warmup": 16, "ms_per_step": live["span_s"] * 1e3 / args.requests, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"serve: 16 resident files x {args.file_records} records (GEX/ATAC), {args.requests} "
                               f"requests of log-uniform 64 KB-512 MB compressed ranges, Poisson {rate:.1f}/s "
                               f"({'80% of saturation' if not args.rate else 'given'}), 40 GB HBM budget, seed 4",
                   "offered_gbs": rate * mean_bytes / 1e9, "mean_request_inflated_bytes": mean_bytes,
                   "inflated_bytes_requested": total, "small_requests": n_small, "generate_s": round(gen_s, 1),
                   "step_bytes": server.long_step_bytes, "short_step_bytes": server.short_step_bytes,
                   "slice_bytes": server.slice_bytes},
        "served": live, "saturation": sat, "plain_sequential": plain,
        "served_vs_saturation": live["throughput_gbs"] / sat["throughput_gbs"],
        "clocks": clocks,
    }), flush=True)


def run_bai(args):
    """Region access through a BAI index on the GEX file of the default workload: the index built on the
    device, then random regions (log-uniform 1 kb-10 Mb) fetched one at a time (decode of the members
    that hold them, records overlapping the region kept); latency percentiles and records/s."""
    import numpy as np
    import torch

    from cubam_b200 import bai, serve

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    args.config = "gex"
    cfg, n, path, gen_s = ensure_file(args, 0, None)
    rf = serve.ResidentFile.load(path)
    torch.cuda.synchronize()
    bai.build(rf)
    torch.cuda.synchronize()
    t = time.perf_counter()
    idx = bai.build(rf)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t
    raw = idx.to_bytes()
    rng = np.random.default_rng(9)
    lengths = rf.header.lengths
    regions = []
    for _ in range(args.requests):
        r = int(rng.integers(len(lengths)))
        size = int(np.exp(rng.uniform(np.log(1e3), np.log(1e7))))
        beg = int(rng.integers(0, max(int(lengths[r]) - size, 1)))
        regions.append((r, beg, beg + size))
    for r, b, e in regions[:10]:
        bai.fetch(rf, idx, r, b, e)
    torch.cuda.synchronize()
    lat, recs = [], 0
    t0 = time.perf_counter()
    for r, b, e in regions:
        t = time.perf_counter()
        res = bai.fetch(rf, idx, r, b, e)
        torch.cuda.synchronize()
        lat.append((time.perf_counter() - t) * 1e3)
        recs += len(res)
    span = time.perf_counter() - t0
    lat = np.array(lat)
    print(json.dumps({
        "metric": "BAM region fetch through a BAI index on 1 B200", "value": recs / span, "unit": "records/s",
        "n_gpus": 1, "steps": len(regions), "warmup": 10, "ms_per_step": span * 1e3 / len(regions),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"{cfg.name}: {n} records; {len(regions)} regions of log-uniform 1 kb-10 Mb, seed 9"},
        "index": {"build_s": build_s, "bytes": len(raw), "refs": len(idx.refs)},
        "fetch_ms": {"p50": float(np.percentile(lat, 50)), "p95": float(np.percentile(lat, 95)),
                     "p99": float(np.percentile(lat, 99))},
        "records": recs,
    }), flush=True)


def _zlib_members(chunk: bytes) -> int:
    from oracle import bgzf_writer_oracle as W

    return len(W.bgzf_compress(chunk, 6)[0])


def run_write(args):
    """The BGZF writer (``cubam_b200.bgzf._bgzf_compress``) on BAM bytes: the inflated records of the
    synthetic GEX file (100,000 records), tiled on the device to ``--write-gb`` GB.  Copies repeat 25 MB
    apart, beyond DEFLATE's 32 KiB window, so each 65,280-byte block compresses as in the original
    file.  value: input GB/s with the input resident in HBM; e2e: the same from pinned host memory
    with the H2D copy of the input and the D2H copy of the members in each step; cpu_baseline: zlib
    level 6 (htslib's default) through the CPU oracle on all host cores, on the same bytes."""
    import multiprocessing as mp

    if int(os.environ.get("RANK", "0")) != 0:
        return  # one GPU: rank 0 alone runs it
    cores = os.cpu_count() or 1
    pool = None
    if not args.no_cpu:  # started, and its workers up, before any GPU call and any timing
        pool = mp.get_context("spawn").Pool(cores)
        pool.map(_zlib_members, [b"warm"] * cores)
    from cubam_b200 import synth

    base = Path(args.workdir or ("/dev/shm" if Path("/dev/shm").exists() else "/tmp"))
    n_rec = args.records or 100_000
    path = base / f"cubam_bench_write_gex_{n_rec}.bam"
    if not path.exists():
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        synth.write_bam(tmp, "gex", n_records=n_rec)
        tmp.replace(path)
    import torch

    from cubam_b200 import _lib, bgzf, bgzf_writer
    from cubam_b200.bgzf import BLOCK_DATA, _bgzf_compress

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    comp = torch.frombuffer(bytearray(path.read_bytes()), dtype=torch.uint8).cuda()
    one, _ = bgzf._inflate_blocks(comp, True)
    copies = max(1, int(args.write_gb * 1e9 // one.numel()))
    data = one.repeat(copies)
    nbytes = int(data.numel())
    del comp
    for _ in range(max(args.warmup, 0)):
        out = _bgzf_compress(data, args.level)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        time.sleep(2.0)  # the sampler's start-up, which stalled host syncs of a short timed region
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(args.steps):
            out = _bgzf_compress(data, args.level)
        stop.record()
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / args.steps
    out_bytes = int(out.numel())
    n_spans = (nbytes + BLOCK_DATA - 1) // BLOCK_DATA
    calls = -(-n_spans // bgzf_writer.SPANS_PER_CALL)

    # the native call alone (k_deflate + k_offsets + k_pack) on one batch of spans, buffers made once
    m = min(n_spans, bgzf_writer.SPANS_PER_CALL)
    off = torch.arange(m, dtype=torch.int64, device="cuda") * BLOCK_DATA
    size = torch.full((m,), BLOCK_DATA, dtype=torch.int64, device="cuda")
    size[-1] = min(BLOCK_DATA, nbytes - (m - 1) * BLOCK_DATA)
    ws = torch.empty(_lib.lib.cb_deflate_workspace_bytes(m), dtype=torch.uint8, device="cuda")
    cap = int(size.sum()) + 36 * m
    o = torch.empty(cap, dtype=torch.uint8, device="cuda")
    oo, osz = torch.empty(m, dtype=torch.int64, device="cuda"), torch.empty(m, dtype=torch.int64, device="cuda")
    summ = torch.zeros(32, dtype=torch.uint8, device="cuda")
    strm = torch.cuda.current_stream().cuda_stream

    def native():
        _lib.check(_lib.lib.cb_deflate_spans(data.data_ptr(), off.data_ptr(), size.data_ptr(), m, args.level, 1,
                                             o.data_ptr(), cap, oo.data_ptr(), osz.data_ptr(), None, summ.data_ptr(),
                                             ws.data_ptr(), ws.numel(), strm), "cb_deflate_spans")

    for _ in range(3):
        native()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    a.record()
    for _ in range(reps):
        native()
    b.record()
    torch.cuda.synchronize()
    native_ms = a.elapsed_time(b) / reps
    in_native = int(size.sum())
    out_native = int(bgzf.read_struct(summ, _lib.DeflateSummary).total)
    peak, peak_kind = peaks()
    achieved = (in_native + out_native) / (native_ms / 1e3) / 1e9

    e2e = None
    if not args.no_e2e:
        host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        host.copy_(data)
        back = torch.empty(out_bytes + (1 << 20), dtype=torch.uint8, pin_memory=True)
        steps = max(args.e2e_steps, 1)
        for _ in range(1):
            d = host.cuda(non_blocking=True)
            r = _bgzf_compress(d, args.level)
            back[: r.numel()].copy_(r)
        torch.cuda.synchronize()
        a.record()
        d2h = 0
        for _ in range(steps):
            d = host.cuda(non_blocking=True)
            r = _bgzf_compress(d, args.level)
            back[: r.numel()].copy_(r)
            d2h = int(r.numel())
        b.record()
        torch.cuda.synchronize()
        e_ms = a.elapsed_time(b) / steps
        e2e = {"value": nbytes / (e_ms / 1e3) / 1e9, "unit": "GB/s", "ms_per_step": e_ms,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": d2h,
               "path": "pinned host bytes -> _bgzf_compress -> pinned host members"}

    cpu = None
    if not args.no_cpu:
        sample = one.cpu().numpy().tobytes()
        chunk = 16 * BLOCK_DATA
        parts = [sample[i : i + chunk] for i in range(0, len(sample), chunk)]
        t = time.perf_counter()
        z6 = sum(pool.map(_zlib_members, parts))
        secs = time.perf_counter() - t
        cpu = {"value": len(sample) / secs / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
               "sample": f"the {len(sample) / 1e6:.0f} MB of the file once (one copy of the tiled input): "
                         f"BGZF members with zlib level 6 in {secs:.2f} s",
               "ratio": z6 / len(sample)}
    if pool:
        pool.terminate()
    print(json.dumps({
        "metric": "BGZF compress GB/s (uncompressed input) on 1 B200", "value": nbytes / (ms / 1e3) / 1e9,
        "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"inflated GEX BAM bytes ({n_rec} records, {one.numel()} bytes) x {copies} copies",
                   "input_bytes": nbytes, "level": args.level, "spans": n_spans, "native_calls_per_step": calls,
                   "l2": "inputs larger than L2 (no flush)"},
        "ratio": out_bytes / nbytes,
        "roofline": {"bound": "hbm", "kernel": "k_deflate", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic": "input bytes read + member bytes written per native call "
                                    "(k_deflate + k_offsets + k_pack, k_deflate dominant)",
                     "native_ms": native_ms, "native_spans": m, "traffic": None},
        "clocks": clk.summary(),
        "gpu_launches": 3 * calls * args.steps,
        **({"e2e": e2e} if e2e else {}),
        **({"cpu_baseline": cpu} if cpu else {}),
    }), flush=True)


def main():
    args = parse()
    if args.config == "write":
        run_write(args)
    elif args.config == "bai":
        run_bai(args)
    elif args.config == "serve":
        run_serve(args)
    elif args.config == "uneven":
        run_uneven(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
