"""Benchmark: BCn encode throughput on B200 (Mpixel/s).

Workload of the contract line (one "step"): the 2048x2048 RGBA8
texture-with-alpha image encoded as BC7 (alpha_basic profile), BC3 and BC4 (R
channel), plus BC5 of a 2048x2048 normal map -- 4 x 4.19 Mpx of encoded
texels per step. Seeded synthetic content (block_compression_b200/synthetic.py);
no dataset is involved.

value: encoded Mpixel/s over the whole job (all ranks), device-resident
  inputs, CUDA-event timed per step with an L2 flush (a 256 MiB write)
  before every step.
e2e:   the same metric through the public host-buffer entry points
  (bc_compress_rgba8 with pinned host buffers: H2D copy, kernels, D2H copy,
  synchronize), as a reference user would call compress_rgba8; the step's
  four textures are encoded from four host threads (e2e.sequential_value:
  the four calls one after another). Each leg times the K steps three times
  and reports the median (e2e.repeats lists all three).

The same line carries the other workloads of the metric, each timed with CUDA
events (L2 flushed before every launch), with its own roofline, CPU baseline
and full bit-exact check against the CPU oracle:
  c1  BC1 encode + decode of the 1024x1024 image (HBM roofline; also at
      8192x8192, where the launch is long enough for the bound to show);
  c3  BC6H basic encode of the 1024x1024 RGBA16F HDR image (FP32 issue roofline);
  c4  64 textures with full mip chains, BC1/BC5/BC7 round-robin: the batched
      CUDA graph against per-task launches, per variant group too.

--impl reference times the reference algorithm on the host CPU (the C++
restatement of the Rust encoder in oracle/, all host threads) on the full
2048x2048 workload every step; the GPU arm's `cpu_baseline` is the same
measurement, plus a single-thread figure on a row sample.

Multi-GPU: one process per GPU. Under torchrun the ranks come from the
environment; `--gpus N` without it starts the N replica processes itself.
Each rank encodes its own copy of the workload (independent textures, no data
exchange); max-over-ranks device time, weak scaling.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = H = 2048
# Algorithmic work per 4x4 block: FP32 operations of the reference encoder
# (add/sub/mul/div/sqrt/abs/min/max/compare/convert), measured with the
# op-counting build of the CPU restatement (`python -m oracle.count_ops`,
# 2048 sampled blocks of each workload's content).
OPS_PER_BLOCK = {"bc7_alpha_basic": 354530.4, "bc3": 1155.0, "bc4": 101.4, "bc5": 202.3,
                 "bc6h_basic": 77119.8, "bc1": 954.3}
SMS, FP32_LANES_PER_SM = 148, 128
# DRAM bytes (read + write) of one BC7 encode of the 2048x2048 workload, summed
# over the pipeline's launches, from an ncu capture with the L2 left warm
# between launches (--cache-control none), as in a real encode.
BC7_DRAM_BYTES_PER_LAUNCH = 137.4e6
METRIC = "BC7/BC6H/BC1 encode Mpixel/s on 1 B200 at reference PSNR; batched vs plain vs CPU"
WORKLOAD = "2048x2048 RGBA8 alpha texture: BC7 alpha_basic + BC3 + BC4(R); 2048x2048 normal map: BC5"
A7 = [2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 12, 8, 8, 0, 2, 4]  # BC7Settings::alpha_basic()
B6 = [0, 0, 2, 2, 4]                                               # BC6HSettings::basic()
E2E_REPEATS = 3  # timed repetitions of each end-to-end leg (median reported)


def config_dict():
    """The `config` of both arms' lines (identical keys and values)."""
    return {"workload": WORKLOAD, "px_per_step": 4 * W * H, "bc7_settings": "alpha_basic",
            "l2": "GPU arm: flushed (256 MiB write) before each step; CPU arm: not applicable",
            "seeds": {"image": 2, "normal_map": 2}}


def _synthetic():
    """The seeded generators, loaded by file path: importing the package would
    load libbcn_b200.so, which the CPU arm must not map."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bcn_synthetic",
                                                  os.path.join(ROOT, "block_compression_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons of this rank's GPU during the timed
    region. NVML, sampled every 2 ms on a thread and once more at the start
    and at the end (so a region shorter than the interval still has
    samples), the GPU found by its PCI address (NVML numbers every GPU of
    the machine, not the visible ones); `nvidia-smi -lms 100` by UUID as the
    fallback."""

    REASON_BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
                   "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.nv = None
        self.h = None
        self.samples = []
        self.max_mhz = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.index)
        for fmt in ("%08X:%02X:%02X.0", "%04X:%02X:%02X.0"):
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(
                    (fmt % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)).encode())
            except pynvml.NVMLError:
                continue
        raise RuntimeError("no NVML device at the GPU's PCI address")

    def _sample(self):
        sm = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
        reasons = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        self.samples.append((float(sm), int(reasons)))

    def _loop(self):
        while not self.stop.wait(0.002):
            try:
                self._sample()
            except Exception:
                return

    def __enter__(self):
        try:
            self.nv, self.h = self._nvml_handle()
            self.max_mhz = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            self._sample()
            self.stop = threading.Event()
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.h = None
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            sel = str(self.index)
            try:
                import torch
                sel = "GPU-" + str(torch.cuda.get_device_properties(self.index).uuid)
            except Exception:
                pass
            self.proc = subprocess.Popen(["nvidia-smi", "-i", sel, "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.h is not None:
            self.stop.set()
            self.t.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.samples:
            sm = [x for x, _ in self.samples]
            reasons = sorted(n for n, bit in self.REASON_BITS.items() if any(r & bit for _, r in self.samples))
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(sm), "source": "nvml"}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(ms, pg, device):
    """The largest of every rank's time (each rank passes its own); `pg` is
    torch.distributed (or None for one process)."""
    if pg is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def bc7_kernel_count(s):
    """Kernels one BC7 encode launches (bc7_encode.cu run_pipeline): prep, a
    refine per mode with candidates (0, 2, 1, 3, 7) and a search per mode,
    modes 1 and 3 sharing one search launch, the three mode-4/5 launches when
    rotations are searched, mode 6, select."""
    ms = [bool(x) for x in s.mode_selection]
    run13 = ms[1] and bool(s.fast_skip_threshold_mode1 or s.fast_skip_threshold_mode3)
    run7 = ms[1] and bool(s.fast_skip_threshold_mode7)
    counts = [16 if ms[0] else 0, 64 if (ms[0] and not s.skip_mode2) else 0,
              s.fast_skip_threshold_mode1 if run13 else 0, s.fast_skip_threshold_mode3 if run13 else 0,
              s.fast_skip_threshold_mode7 if run7 else 0]
    nrefine = sum(1 for c in counts if c)
    nsearch = nrefine - (1 if counts[2] and counts[3] else 0)
    nrot = max(0, int(s.channels) - int(s.mode45_channel0)) if ms[2] else 0
    return 1 + nsearch + nrefine + (3 if nrot else 0) + (1 if ms[3] else 0) + 1


def job_mpx_s(world, px_per_rank_step, steps, ms):
    """Whole-job throughput of a weak-scaling run: every rank encodes
    px_per_rank_step pixels per step; ms is the max-over-ranks time."""
    return world * px_per_rank_step * steps / (ms / 1e3) / 1e6


# ---- CPU side: the reference encoder restated in C++ (oracle/) ------------------------


def c2_inputs(syn):
    return {"img": syn.config2_image(seed=2, size=W), "nrm": syn.normal_map(seed=2, size=W)}


C2_JOBS = [("bc7_alpha_basic", 6, "img", A7), ("bc3", 2, "img", None), ("bc4", 3, "img", None),
           ("bc5", 4, "nrm", None)]


def cpu_c2_step(oracle, inputs, threads):
    """One step of the contract workload on the CPU: the four full 2048x2048
    encodes. Returns (seconds, {job: blocks})."""
    outs = {}
    t0 = time.perf_counter()
    for name, vid, key, s in C2_JOBS:
        outs[name] = oracle.compress_rgba8(vid, inputs[key], W, H, settings=s, threads=threads)
    return time.perf_counter() - t0, outs


def row_sample(img, every=16):
    """Every `every`-th row of 4x4 blocks of an image, stacked: a sample
    spread over the whole image (2048 x 128 for the 2048x2048 inputs)."""
    rows = [img[y:y + 4] for y in range(0, img.shape[0], 4 * every)]
    import numpy as np
    return np.ascontiguousarray(np.concatenate(rows, axis=0))


def cpu_c2_single_thread(oracle, inputs):
    """Mpixel/s of the contract workload on one host thread, on the block-row
    sample of each input."""
    sample = {k: row_sample(v) for k, v in inputs.items()}
    h = sample["img"].shape[0]
    t0 = time.perf_counter()
    for name, vid, key, s in C2_JOBS:
        oracle.compress_rgba8(vid, sample[key], W, h, settings=s, threads=1)
    return 4 * W * h / (time.perf_counter() - t0) / 1e6


def cpu_reference(args, world, rank):
    """Reference arm: the reference's encoder restated in C++ (oracle/), all
    host threads, on the full contract workload every step."""
    if rank != 0:
        return
    import oracle
    syn = _synthetic()
    inputs = c2_inputs(syn)
    threads = os.cpu_count()
    for _ in range(max(1, args.warmup)):
        cpu_c2_step(oracle, inputs, threads)
    times = [cpu_c2_step(oracle, inputs, threads)[0] for _ in range(args.steps)]
    t = sum(times) / len(times)
    value = 4 * W * H / t / 1e6
    sample = "the full workload every step: BC7 alpha_basic, BC3, BC4 of the 2048x2048 image, BC5 of the normal map"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_dict(),
        "cpu_baseline": {"value": value, "unit": "Mpixel/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Mpixel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- GPU side ---------------------------------------------------------------------------


class DeviceTimer:
    """CUDA-event times of launches on the current stream, each preceded by
    an L2 flush (a 256 MiB write, twice the L2)."""

    def __init__(self, torch, dev):
        self.torch = torch
        self.flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def time(self, fn, steps, warmup=3):
        torch = self.torch
        stream = torch.cuda.current_stream()
        out = []
        for i in range(warmup + steps):
            self.flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            if i >= warmup:
                out.append(a.elapsed_time(b))
        return sum(out) / len(out)


def hbm_roofline(kernel, nbytes, ms, peaks, src):
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"kernel": kernel, "bound": "hbm", "unit": "GB/s", "achieved": gbs, "peak": peaks["hbm_gbs"],
            "frac": gbs / peaks["hbm_gbs"], "traffic": None, "algorithmic_bytes_per_launch": nbytes,
            "ms_per_launch": ms, "peak_source": "hbm_gbs (%s)" % src}


def issue_roofline(kernel, ops_per_block, nblocks, ms, peaks, src):
    peak = SMS * FP32_LANES_PER_SM * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    achieved = ops_per_block * nblocks / (ms / 1e3) / 1e12
    return {"kernel": kernel, "bound": "fp32", "unit": "TFLOP/s", "achieved": achieved, "peak": peak,
            "frac": achieved / peak, "algorithmic_ops_per_block": ops_per_block, "ms_per_launch": ms,
            "peak_source": "148 SMs x 128 FP32 lanes x %s sm_max_mhz (%s)" % (peaks.get("sm_max_mhz"), src)}


def bench_c1(bcn, torch, dev, timer, syn, oracle, steps, peaks, src, verify, cpu):
    """BC1 encode + decode of the 1024x1024 image (config 1), and the same
    kernels on the image tiled to 8192x8192 (inputs far beyond L2)."""
    import numpy as np
    V = bcn.CompressionVariant
    img = syn.config1_image(seed=1, size=1024)
    res = {"workload": "BC1 encode + decode, 1024x1024 RGBA8 (gradients, value noise, 32 triangles), seed 1"}
    for size, reps in ((1024, 1), (8192, 8)):
        src_t = torch.from_numpy(np.tile(img, (reps, reps, 1)) if reps > 1 else img).to(dev)
        blocks = torch.zeros(V.BC1.blocks_byte_size(size, size), dtype=torch.uint8, device=dev)
        out = torch.zeros(size * size * 4, dtype=torch.uint8, device=dev)
        enc_ms = timer.time(lambda: bcn.encode.compress_rgba8(V.BC1, src_t, blocks, size, size, size * 4), steps)
        dec_ms = timer.time(lambda: bcn.decode.decompress_blocks_as_rgba8(V.BC1, size, size, blocks, out), steps)
        nbytes = size * size * 4 + (size // 4) ** 2 * 8
        key = "" if size == 1024 else "_8192"
        res["encode_mpx_s" + key] = size * size / enc_ms / 1e3
        res["decode_mpx_s" + key] = size * size / dec_ms / 1e3
        res["roofline_encode" + key] = hbm_roofline("bc15_encode_kernel<BC1>", nbytes, enc_ms, peaks, src)
        res["roofline_decode" + key] = hbm_roofline("bc15_decode_kernel<BC1>", nbytes, dec_ms, peaks, src)
        if size == 1024:
            res["roofline_issue_encode"] = issue_roofline("bc15_encode_kernel<BC1>", OPS_PER_BLOCK["bc1"],
                                                          (size // 4) ** 2, enc_ms, peaks, src)
            got_b, got_px = blocks.cpu().numpy(), out.cpu().numpy()
        del src_t, blocks, out
    if verify:
        exp_b = oracle.compress_rgba8(0, img, 1024, 1024)
        res["verified_full"] = bool(np.array_equal(got_b, exp_b) and
                                    np.array_equal(got_px, oracle.decompress_rgba8(0, exp_b, 1024, 1024)))
    if cpu:
        threads = os.cpu_count()
        t0 = time.perf_counter()
        for _ in range(5):
            b = oracle.compress_rgba8(0, img, 1024, 1024, threads=threads)
        te = (time.perf_counter() - t0) / 5
        t0 = time.perf_counter()
        for _ in range(5):
            oracle.decompress_rgba8(0, b, 1024, 1024, threads=threads)
        td = (time.perf_counter() - t0) / 5
        res["cpu_baseline"] = {"value": 1024 * 1024 / te / 1e6, "unit": "Mpixel/s (encode)",
                               "decode_mpx_s": 1024 * 1024 / td / 1e6, "cores": threads, "kind": "port",
                               "sample": "the full 1024x1024 image, 5 passes"}
    return res


def bench_c3(bcn, torch, dev, timer, syn, oracle, steps, peaks, src, verify, cpu):
    """BC6H basic encode of the 1024x1024 RGBA16F HDR image (config 3)."""
    import numpy as np
    s6 = bcn.BC6HSettings.basic()
    v = bcn.CompressionVariant.BC6H(s6)
    hdr = syn.config3_hdr(seed=3, size=1024)
    src_t = torch.from_numpy(hdr.view(np.int16)).to(dev)
    blocks = torch.zeros(v.blocks_byte_size(1024, 1024), dtype=torch.uint8, device=dev)
    ms = timer.time(lambda: bcn.encode.compress_rgba16(v, src_t, blocks, 1024, 1024, 1024 * 4), steps)
    res = {"workload": "BC6H basic encode, 1024x1024 RGBA16F HDR (log-uniform 2^-8..2^8, 2% spikes), seed 3",
           "encode_mpx_s": 1024 * 1024 / ms / 1e3,
           "roofline": issue_roofline("bc6h_encode_kernel", OPS_PER_BLOCK["bc6h_basic"], 256 * 256, ms, peaks, src)}
    got = blocks.cpu().numpy()
    from block_compression_b200 import metrics
    res["log_luminance_rmse"] = metrics.log_luminance_rmse(src_t, blocks, 1024, 1024)
    if verify or cpu:
        threads = os.cpu_count()
        t0 = time.perf_counter()
        exp = oracle.compress_rgba16(hdr.view(np.uint16), 1024, 1024, B6, threads=threads)
        tc = time.perf_counter() - t0
        if verify:
            res["verified_full"] = bool(np.array_equal(got, exp))
            # FP64 recomputation of every block's squared error, ours against
            # the reference's blocks, and the reference's log-luminance RMSE
            exp_t = torch.from_numpy(exp).to(dev)
            sse_g = torch.zeros(256 * 256, dtype=torch.float64, device=dev)
            sse_r = torch.zeros(256 * 256, dtype=torch.float64, device=dev)
            metrics.bc6h_error(src_t, blocks, 1024, 1024, block_sse=sse_g)
            metrics.bc6h_error(src_t, exp_t, 1024, 1024, block_sse=sse_r)
            excess = ((sse_g - sse_r) / sse_r.clamp_min(1e-300)).max().item()
            res["quality"] = {
                "log_luminance_rmse_reference": metrics.log_luminance_rmse(src_t, exp_t, 1024, 1024),
                "blocks_bit_identical": float((got.reshape(-1, 16) == exp.reshape(-1, 16)).all(1).mean()),
                "max_block_sse_excess_rel": max(0.0, excess),
                "metric": "RGB squared error and log2 Rec.709 luminance error in f64 (bc_bc6h_error_device)"}
        if cpu:
            res["cpu_baseline"] = {"value": 1024 * 1024 / tc / 1e6, "unit": "Mpixel/s", "cores": threads,
                                   "kind": "port", "sample": "the full 1024x1024 image"}
    return res


def bench_c4(bcn, torch, dev, syn, oracle, steps, verify, cpu, textures=64):
    """Config 4: `textures` RGBA8 textures (sides from {16, 20, ..., 4096}),
    full GPU-made box-filtered mip chains, BC1 / BC5 / BC7 alpha_basic
    round-robin; per-task launches against the batched CUDA graph with the
    autotuned launch shape, for all tasks and per variant group."""
    import numpy as np

    from block_compression_b200 import mips
    V = bcn.CompressionVariant
    variants = [V.BC1, V.BC5, V.BC7(bcn.BC7Settings.alpha_basic())]
    shapes = syn.config4_textures(seed=4, count=textures)
    chains = [mips.generate_mip_chain(syn.rgba8_textured_torch(4000 + i, h, w, dev)) for i, (h, w) in
              enumerate(shapes)]
    tasks, total = [], 0
    for i, chain in enumerate(chains):
        v = variants[i % 3]
        for li, lv in enumerate(chain):
            n = v.blocks_byte_size(lv.padded_width, lv.padded_height)
            tasks.append((lv, v, total, n, li))
            total += n
    torch.cuda.synchronize()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def run(sub, out, batched, reps):
        c = bcn.GpuBlockCompressor()
        times = []
        if batched:
            for lv, v, off, n, _ in sub:
                c.add_compression_task(v, lv.data, lv.padded_width, lv.padded_height, out, blocks_offset=off)
            t0 = time.perf_counter()
            b = c.create_batch(autotune=True)
            torch.cuda.synchronize()
            tune_s = time.perf_counter() - t0
        for i in range(1 + reps):
            if not batched:
                for lv, v, off, n, _ in sub:
                    c.add_compression_task(v, lv.data, lv.padded_width, lv.padded_height, out, blocks_offset=off)
            a, z = ev(), ev()
            a.record()
            b.launch() if batched else c.compress()
            z.record()
            torch.cuda.synchronize()
            if i:
                times.append(a.elapsed_time(z))
        extra = {}
        if batched:
            extra = {"tune": b.tune.as_dict(), "autotune_s": tune_s}
            b.close()
        return sum(times) / len(times), extra

    reps = max(2, min(steps, 5))
    out_p = torch.zeros(total, dtype=torch.uint8, device=dev)
    out_b = torch.zeros(total, dtype=torch.uint8, device=dev)
    px = sum(lv.padded_width * lv.padded_height for lv, _, _, _, _ in tasks)
    pm, _ = run(tasks, out_p, False, reps)
    bm, extra = run(tasks, out_b, True, reps)
    res = {"workload": "%d RGBA8 textures, sides in {16..4096}, full mip chains, BC1/BC5/BC7 alpha_basic "
                       "round-robin, seed 4" % textures,
           "tasks": len(tasks), "encoded_mpx": px / 1e6, "plain_ms": pm, "batched_ms": bm,
           "plain_mpx_s": px / pm / 1e3, "batched_mpx_s": px / bm / 1e3, "batched_over_plain": pm / bm,
           "outputs_identical": bool(torch.equal(out_p, out_b))}
    res.update(extra)
    groups = {}
    for gname, keep in (("bc7", lambda v: v.id == 6), ("bc1_bc5", lambda v: v.id != 6)):
        sub = [t for t in tasks if keep(t[1])]
        gpx = sum(lv.padded_width * lv.padded_height for lv, _, _, _, _ in sub)
        gp, _ = run(sub, out_p, False, reps)
        gb, _ = run(sub, out_b, True, reps)
        groups[gname] = {"tasks": len(sub), "encoded_mpx": gpx / 1e6, "plain_ms": gp, "batched_ms": gb,
                         "batched_over_plain": gp / gb}
    res["by_variant"] = groups
    if verify or cpu:
        # every level from the 4th down (a spread sample of the chains, about
        # 1/48 of the pixels): the oracle's blocks against the batched output
        # and the oracle's time per variant, scaled by each variant's pixels
        got = out_b.cpu().numpy()
        threads = os.cpu_count()
        t_v, px_v, all_px_v, ok = {}, {}, {}, True
        for lv, v, off, n, li in tasks:
            all_px_v[v.id] = all_px_v.get(v.id, 0) + lv.padded_width * lv.padded_height
            if li < 3:
                continue
            img = lv.data.cpu().numpy()
            s = v.settings.as_list() if v.settings is not None else None
            t0 = time.perf_counter()
            exp = oracle.compress_rgba8(v.id, img, lv.padded_width, lv.padded_height, settings=s, threads=threads)
            t_v[v.id] = t_v.get(v.id, 0.0) + time.perf_counter() - t0
            px_v[v.id] = px_v.get(v.id, 0) + lv.padded_width * lv.padded_height
            ok = ok and bool(np.array_equal(got[off:off + n], exp))
        if verify:
            res["verified_sample"] = ok and res["outputs_identical"]
        if cpu:
            est = sum(t_v[k] * all_px_v[k] / px_v[k] for k in t_v)
            res["cpu_baseline"] = {"value": px / est / 1e6, "unit": "Mpixel/s", "cores": threads, "kind": "port",
                                   "sample": "mip levels 3 and below of every texture (%.1f Mpx), time scaled per "
                                             "variant by its pixel count" % (sum(px_v.values()) / 1e6)}
    del chains, out_p, out_b
    return res


def gpu_bench(args, world, rank, local):
    import numpy as np
    import torch

    import block_compression_b200 as bcn
    syn = _synthetic()

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        # rank 0 verifies the outputs and runs the c1/c3/c4 workloads while the
        # other ranks wait at the final barrier: the timeout leaves room for that
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    V = bcn.CompressionVariant
    s7 = bcn.BC7Settings.alpha_basic()
    jobs = [("bc7_alpha_basic", V.BC7(s7), "img"), ("bc3", V.BC3, "img"), ("bc4", V.BC4, "img"), ("bc5", V.BC5, "nrm")]
    inputs = c2_inputs(syn)
    img_np, nrm_np = inputs["img"], inputs["nrm"]
    srcs = {"img": torch.from_numpy(img_np).to(dev), "nrm": torch.from_numpy(nrm_np).to(dev)}
    outs = {name: torch.zeros(v.blocks_byte_size(W, H), dtype=torch.uint8, device=dev) for name, v, _ in jobs}
    timer = DeviceTimer(torch, dev)
    flush = timer.flush
    stream = torch.cuda.current_stream(dev)
    import ctypes
    sp = ctypes.c_void_p(stream.cuda_stream)

    def run_step(evs=None):
        for i, (name, v, key) in enumerate(jobs):
            if evs is not None:
                evs[i][0].record(stream)
            bcn.encode.compress_rgba8(v, srcs[key], outs[name], W, H, W * 4, stream=sp)
            if evs is not None:
                evs[i][1].record(stream)

    for _ in range(max(3, args.warmup)):
        flush.fill_(1)
        run_step()
    torch.cuda.synchronize()

    step_ms, per_job = [], {name: [] for name, _, _ in jobs}
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)  # evict the inputs from L2 (126 MB) before each step
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in jobs]
            run_step(evs)
            torch.cuda.synchronize()
            t = 0.0
            for (name, _, _), (a, b) in zip(jobs, evs):
                ms = a.elapsed_time(b)
                per_job[name].append(ms)
                t += ms
            step_ms.append(t)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    total_ms = max_over_ranks(sum(step_ms), pg, dev)
    px_per_step = 4 * W * H
    value = job_mpx_s(world, px_per_step, args.steps, total_ms)

    # e2e through the host entry points with pinned host buffers
    pin_img = torch.from_numpy(img_np).pin_memory()
    pin_nrm = torch.from_numpy(nrm_np).pin_memory()
    host_src = {"img": pin_img.numpy(), "nrm": pin_nrm.numpy()}
    pin_out = {name: torch.zeros(v.blocks_byte_size(W, H), dtype=torch.uint8).pin_memory() for name, v, _ in jobs}
    host_out = {k: t.numpy() for k, t in pin_out.items()}

    def e2e_sequential():
        for name, v, key in jobs:
            bcn.encode.compress_rgba8(v, host_src[key], host_out[name], W, H, W * 4)

    # The step's four textures are encoded by four host threads, one per
    # texture, each with a blocking host-buffer call -- as an application
    # encoding several textures does. The library's host entry points keep
    # their staging buffers and streams per thread, so one texture's copies
    # overlap another's kernels. Each worker thread has the rank's device
    # current and keeps its texture, so its buffers are made once, in the
    # warm-up steps.
    from concurrent.futures import ThreadPoolExecutor
    workers = [ThreadPoolExecutor(1, initializer=torch.cuda.set_device, initargs=(local,)) for _ in jobs]

    def e2e_parallel():
        futs = [wk.submit(bcn.encode.compress_rgba8, v, host_src[key], host_out[name], W, H, W * 4)
                for wk, (name, v, key) in zip(workers, jobs)]
        for f in futs:
            f.result()

    def timed(step_fn):
        for _ in range(2):
            step_fn()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step_fn()
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3), pg, dev)

    # Three timed repetitions of the K steps per leg, interleaved, and their
    # median: host threads and the shared PCIe link make single runs of the
    # threaded leg vary by several percent. All repetitions are reported.
    seq_reps, par_reps = [], []
    for _ in range(E2E_REPEATS):
        seq_reps.append(timed(e2e_sequential))
        par_reps.append(timed(e2e_parallel))
    e2e_seq_ms = sorted(seq_reps)[len(seq_reps) // 2]
    e2e_ms = sorted(par_reps)[len(par_reps) // 2]
    for wk in workers:
        wk.shutdown()
    e2e_value = job_mpx_s(world, px_per_step, args.steps, e2e_ms)
    e2e_seq_value = job_mpx_s(world, px_per_step, args.steps, e2e_seq_ms)
    h2d = 3 * img_np.nbytes + nrm_np.nbytes
    d2h = sum(v.blocks_byte_size(W, H) for _, v, _ in jobs)
    if pg:
        pg.barrier()

    if rank == 0:
        import oracle
        peaks, src = _peaks()
        verify = not args.no_verify
        cpu_leg = world == 1 and not args.no_cpu
        # the oracle's outputs of the whole workload: the full bit-exact check
        # of every encoded block, and (one rank, one GPU) the CPU baseline
        cpu, verified = None, None
        if verify or cpu_leg:
            threads = os.cpu_count()
            tc, exp = cpu_c2_step(oracle, inputs, threads)
            verified = {name: bool(np.array_equal(outs[name].cpu().numpy(), exp[name])) for name, _, _ in jobs}
            verified["host_entry_points"] = all(bool(np.array_equal(host_out[name], exp[name])) for name, _, _ in jobs)
            if cpu_leg:
                cpu = {"value": px_per_step / tc / 1e6, "unit": "Mpixel/s", "cores": threads, "kind": "port",
                       "sample": "the full workload (same measurement as the reference arm): BC7 alpha_basic, BC3, "
                                 "BC4 of the 2048x2048 image, BC5 of the normal map",
                       "single_thread": {"value": cpu_c2_single_thread(oracle, inputs), "unit": "Mpixel/s",
                                         "cores": 1, "sample": "every 16th row of blocks of each input (2048x128)"}}
        bc7_ms = sum(per_job["bc7_alpha_basic"]) / len(per_job["bc7_alpha_basic"])
        per_variant = {name: W * H / (sum(ms) / len(ms) / 1e3) / 1e6 for name, ms in per_job.items()}
        nblk = (W // 4) * (H // 4)
        roof = issue_roofline("BC7 encode pipeline (bc7_prep/search/refine/mode45/mode6/select)",
                              OPS_PER_BLOCK["bc7_alpha_basic"], nblk, bc7_ms, peaks, src)
        roof["traffic"] = BC7_DRAM_BYTES_PER_LAUNCH
        hbm = {}
        for name in ("bc3", "bc4", "bc5"):
            ms = sum(per_job[name]) / len(per_job[name])
            nbytes = W * H * 4 + nblk * (8 if name == "bc4" else 16)
            hbm[name] = hbm_roofline("bc15_encode_kernel<%s>" % name.upper(), nbytes, ms, peaks, src)
        extra = {}
        if not args.no_extra:
            extra["c1"] = bench_c1(bcn, torch, dev, timer, syn, oracle, max(3, args.steps), peaks, src, verify,
                                   cpu_leg)
            extra["c3"] = bench_c3(bcn, torch, dev, timer, syn, oracle, max(3, args.steps), peaks, src, verify,
                                   cpu_leg)
            extra["c4"] = bench_c4(bcn, torch, dev, syn, oracle, args.steps, verify, cpu_leg)
        line = {
            "metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(),
            "e2e": {"value": e2e_value, "unit": "Mpixel/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "calls": "bc_compress_rgba8 with pinned host buffers, the step's 4 textures from 4 host threads",
                    "sequential_value": e2e_seq_value,
                    "statistic": "median of %d timed repetitions of the K steps" % E2E_REPEATS,
                    "repeats": [job_mpx_s(world, px_per_step, args.steps, t) for t in par_reps],
                    "sequential_repeats": [job_mpx_s(world, px_per_step, args.steps, t) for t in seq_reps]},
            # our kernels in the timed region: the BC7 pipeline plus one
            # kernel each for BC3, BC4 and BC5, per step
            "gpu_launches": (bc7_kernel_count(s7) + len(jobs) - 1) * args.steps,
            "per_variant_mpx_s": per_variant,
            "roofline": roof, "roofline_hbm_paths": hbm,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "verified_full": verified,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_replicas(n, argv):
    """Starts `n` processes of this script, one per GPU (rank i on GPU i),
    with the rendezvous environment torchrun would set; returns the worst
    exit status. Only rank 0 prints."""
    port = _free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + argv, env=env))
    rcs = [p.wait() for p in procs]
    return max(rcs, key=abs)


def ranks_selftest(args, world, rank):
    """The replica plumbing alone, on the CPU: rendezvous (gloo), barrier,
    max-over-ranks of a per-rank time, the whole-job throughput. Rank 0
    prints one line. Used by the multi-rank CPU test."""
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        my_ms = 10.0 + 5.0 * rank
        ms = max_over_ranks(my_ms, dist, "cpu")
        if rank == 0:
            print(json.dumps({"world": world, "max_ms": ms, "mpx_s": job_mpx_s(world, 4 * W * H, 10, ms)}),
                  flush=True)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def profile_case(args):
    """Runs one encoder on a square synthetic texture for profilers (ncu):
    `--case bc7:512` = BC7 alpha_basic on 512x512. Prints one line of kernel
    timings; it is not a benchmark line."""
    import torch

    import block_compression_b200 as bcn
    from block_compression_b200 import synthetic

    name, size = args.case.split(":")
    size = int(size)
    V = bcn.CompressionVariant
    variants = {"bc1": V.BC1, "bc3": V.BC3, "bc4": V.BC4, "bc5": V.BC5,
                "bc7": V.BC7(bcn.BC7Settings.alpha_basic()), "bc6h": V.BC6H(bcn.BC6HSettings.basic())}
    v = variants[name]
    if name == "bc6h":
        src = torch.from_numpy(synthetic.config3_hdr(seed=3, size=size).view("int16")).cuda()
    else:
        src = torch.from_numpy(synthetic.config2_image(seed=2, size=size)).cuda()
    dst = torch.zeros(v.blocks_byte_size(size, size), dtype=torch.uint8, device="cuda")
    times = []
    for i in range(args.warmup + args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        if name == "bc6h":
            bcn.encode.compress_rgba16(v, src, dst, size, size, size * 4)
        else:
            bcn.encode.compress_rgba8(v, src, dst, size, size, size * 4)
        b.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(a.elapsed_time(b))
    ms = sum(times) / max(1, len(times))
    print(json.dumps({"case": args.case, "ms": ms, "mpx_s": size * size / ms / 1e3}), flush=True)


def batched_mips_bench(args):
    """Batched mixed workload: 64 RGBA8 textures with sides drawn from
    {16, 20, ..., 4096}, each with its full box-filtered mip chain (GPU), BC1 /
    BC5 / BC7 alpha_basic round-robin; the per-task path (one launch sequence
    per texture level) against the batched CUDA graph with the autotuned
    launch shape. Prints one line (not the benchmark contract line)."""
    import torch

    import block_compression_b200 as bcn
    from block_compression_b200 import mips, synthetic

    dev = torch.device("cuda", 0)
    V = bcn.CompressionVariant
    variants = [V.BC1, V.BC5, V.BC7(bcn.BC7Settings.alpha_basic())]
    shapes = synthetic.config4_textures(seed=4, count=args.textures)
    chains = [mips.generate_mip_chain(synthetic.rgba8_textured_torch(4000 + i, h, w, dev)) for i, (h, w) in
              enumerate(shapes)]
    torch.cuda.synchronize()
    tasks, total, px = [], 0, 0
    for i, chain in enumerate(chains):
        v = variants[i % 3]
        for lv in chain:
            n = v.blocks_byte_size(lv.padded_width, lv.padded_height)
            tasks.append((lv, v, total))
            total += n
            px += lv.padded_width * lv.padded_height
    out_plain = torch.zeros(total, dtype=torch.uint8, device=dev)
    out_batch = torch.zeros(total, dtype=torch.uint8, device=dev)

    def add(c, out):
        for lv, v, off in tasks:
            c.add_compression_task(v, lv.data, lv.padded_width, lv.padded_height, out, blocks_offset=off)

    c = bcn.GpuBlockCompressor()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    plain_ms = []
    for i in range(args.warmup + args.steps):
        add(c, out_plain)
        a, b = ev(), ev()
        a.record()
        c.compress()
        b.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            plain_ms.append(a.elapsed_time(b))
    add(c, out_batch)
    t0 = time.perf_counter()
    batch = c.create_batch(autotune=True)
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t0
    batch_ms = []
    for i in range(args.warmup + args.steps):
        a, b = ev(), ev()
        a.record()
        batch.launch()
        b.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            batch_ms.append(a.elapsed_time(b))
    same = bool(torch.equal(out_plain, out_batch))
    pm, bm = sum(plain_ms) / len(plain_ms), sum(batch_ms) / len(batch_ms)
    tune = batch.tune.as_dict()
    batch.close()

    # the same comparison per variant group: BC7 (compute-bound) and BC1/BC5
    groups = {}
    for gname, keep in (("bc7", lambda v: v.id == 6), ("bc1_bc5", lambda v: v.id != 6)):
        sub = [(lv, v, off) for lv, v, off in tasks if keep(v)]
        gpx = sum(lv.padded_width * lv.padded_height for lv, _, _ in sub)
        cg = bcn.GpuBlockCompressor()
        p_ms = []
        for i in range(args.warmup + args.steps):
            for lv, v, off in sub:
                cg.add_compression_task(v, lv.data, lv.padded_width, lv.padded_height, out_plain, blocks_offset=off)
            a, b = ev(), ev()
            a.record()
            cg.compress()
            b.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                p_ms.append(a.elapsed_time(b))
        for lv, v, off in sub:
            cg.add_compression_task(v, lv.data, lv.padded_width, lv.padded_height, out_batch, blocks_offset=off)
        gb = cg.create_batch(autotune=True)
        b_ms = []
        for i in range(args.warmup + args.steps):
            a, b = ev(), ev()
            a.record()
            gb.launch()
            b.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                b_ms.append(a.elapsed_time(b))
        gb.close()
        gp, gbm = sum(p_ms) / len(p_ms), sum(b_ms) / len(b_ms)
        groups[gname] = {"tasks": len(sub), "encoded_mpx": gpx / 1e6, "plain_ms": gp, "batched_ms": gbm,
                         "batched_over_plain": gp / gbm}
    print(json.dumps({
        "workload": "%d RGBA8 textures, sides in {16..4096}, full mip chains, BC1/BC5/BC7 alpha_basic round-robin"
                    % args.textures,
        "tasks": len(tasks), "encoded_mpx": px / 1e6, "plain_ms": pm, "batched_ms": bm,
        "plain_mpx_s": px / pm / 1e3, "batched_mpx_s": px / bm / 1e3, "batched_over_plain": pm / bm,
        "tune": tune, "autotune_s": tune_s, "outputs_identical": same, "by_variant": groups,
    }), flush=True)


def refine_bench(args):
    """Gradient endpoint refinement workload: 8 RGBA8 images of 512x512 (the
    BC1 generator, seeds 100..107), encoded by the plain BC7 encoder (basic
    opaque profile) and by BC1, then 20 Adam steps at lr 0.5 per block with
    keep-if-better. Reports the refinement kernel's time, the PSNR before and
    after (RGB, exact decoded texels) and the share of blocks replaced, with
    the oracle's sequential restatement timed on one image beside it. Prints
    one line (not the benchmark contract line)."""
    import numpy as np
    import torch

    import block_compression_b200 as bcn
    from block_compression_b200 import refine, synthetic

    dev = torch.device("cuda", 0)
    V = bcn.CompressionVariant
    imgs = [synthetic.config1_image(100 + i, 512) for i in range(8)]
    timgs = [torch.from_numpy(im).to(dev) for im in imgs]
    px = 8 * 512 * 512
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    out = {"workload": "8 RGBA8 images 512x512, 20 Adam steps lr 0.5, keep-if-better", "steps": args.steps}
    for name, variant, per in (("bc7_opaque_basic", V.BC7(bcn.BC7Settings.opaque_basic()), 16), ("bc1", V.BC1, 8)):
        orig = []
        for t in timgs:
            b = torch.zeros(variant.blocks_byte_size(512, 512), dtype=torch.uint8, device=dev)
            bcn.encode.compress_rgba8(variant, t, b, 512, 512, 512 * 4)
            orig.append(b)
        work = [b.clone() for b in orig]
        stats = torch.zeros(4, dtype=torch.int64, device=dev)
        times = []
        for i in range(args.warmup + args.steps):
            for w, o in zip(work, orig):
                w.copy_(o)
            stats.zero_()
            torch.cuda.synchronize()
            a, b = ev(), ev()
            a.record()
            if per == 16:
                refine.refine_bc7_images(list(zip(timgs, work)), channels=3, steps=20, lr=0.5, stats=stats)
            else:
                refine.refine_bc1_images(list(zip(timgs, work)), steps=20, lr=0.5, stats=stats)
            b.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                times.append(a.elapsed_time(b))
        s = stats.cpu().tolist()
        ms = sum(times) / len(times)
        psnr = lambda e: 10 * np.log10(255.0 ** 2 / (e / (px * 3)))  # noqa: E731
        res = {"refine_ms": ms, "refine_mpx_s": px / ms / 1e3, "blocks": s[0], "replaced": s[1],
               "replaced_frac": s[1] / max(1, s[0]), "psnr_before": psnr(s[2]), "psnr_after": psnr(s[3]),
               "sq_err_before": s[2], "sq_err_after": s[3]}
        if not args.no_cpu:
            import oracle
            blk = orig[0].cpu().numpy().reshape(-1, per)
            src = oracle.image_blocks(imgs[0], 512, 512)
            t0 = time.perf_counter()
            oracle.refine_blocks("bc7" if per == 16 else "bc1", blk, src, 20, 0.5, 3)
            dt = time.perf_counter() - t0
            res["cpu_port"] = {"mpx_s": 512 * 512 / dt / 1e6, "cores": 1, "sample": "1 image 512x512"}
        out[name] = res
    print(json.dumps(out), flush=True)


def decode_bench(args):
    """Decode bandwidth: each variant's blocks of an NxN image (encoded once by
    the GPU encoders) decoded to RGBA8 (BC6H also to RGBA16F), L2 flushed
    before every timed launch. Algorithmic bytes per launch = block bytes read
    + texel bytes written. Prints one line (not the benchmark contract line)."""
    import torch

    import block_compression_b200 as bcn
    from block_compression_b200 import synthetic

    dev = torch.device("cuda", 0)
    V = bcn.CompressionVariant
    size = args.decode_size
    peaks, src_kind = _peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    img = synthetic.rgba8_textured_torch(9, size, size, dev)
    reps = max(1, size // 1024)
    hdr = torch.from_numpy(synthetic.config3_hdr(seed=3, size=min(size, 1024)).view("int16")).to(dev)
    hdr = hdr.repeat(reps, reps, 1).contiguous()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    out = {"workload": "decode of %dx%d images, L2 flushed per launch" % (size, size), "hbm_peak_gbs": hbm,
           "peak_source": src_kind}
    b6 = V.BC6H(bcn.BC6HSettings.very_fast())
    cases = [("bc1", V.BC1, 0), ("bc2", V.BC2, 0), ("bc3", V.BC3, 0), ("bc4", V.BC4, 0), ("bc5", V.BC5, 0),
             ("bc7_mode6", V.BC7(bcn.BC7Settings.opaque_ultra_fast()), 0),
             ("bc7_mixed_modes", V.BC7(bcn.BC7Settings.alpha_basic()), 0), ("bc6h_rgba8", b6, 0),
             ("bc6h_rgba16f", b6, 1)]
    for name, v, fmt in cases:
        blocks = torch.zeros(v.blocks_byte_size(size, size), dtype=torch.uint8, device=dev)
        if name.startswith("bc6h"):
            bcn.encode.compress_rgba16(v, hdr, blocks, size, size, size * 4)
        else:
            bcn.encode.compress_rgba8(v, img, blocks, size, size, size * 4)
        dst = torch.empty(size * size * 4, dtype=torch.int16 if fmt else torch.uint8, device=dev)
        dec = bcn.decode.decompress_blocks_as_rgba16f if fmt else bcn.decode.decompress_blocks_as_rgba8
        times = []
        for i in range(args.warmup + args.steps):
            flush.fill_(1)
            a, b = ev(), ev()
            a.record()
            dec(v, size, size, blocks, dst)
            b.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                times.append(a.elapsed_time(b))
        ms = sum(times) / len(times)
        # BC6H to RGBA16F writes the RGB triplets only (the reference's layout)
        written = dst.numel() * dst.element_size() * (3 / 4 if fmt else 1)
        nbytes = blocks.numel() + written
        gbs = nbytes / ms / 1e6
        out[name] = {"ms": ms, "gb_s": gbs, "frac_hbm": gbs / hbm, "bytes_per_launch": int(nbytes),
                     "mpx_s": size * size / ms / 1e3}
    print(json.dumps(out), flush=True)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline legs")
    ap.add_argument("--no-verify", action="store_true", help="skip the bit-exact checks against the oracle")
    ap.add_argument("--no-extra", action="store_true", help="only the contract workload (no c1/c3/c4 objects)")
    ap.add_argument("--case", default=None, help="profiling case VARIANT:SIZE, e.g. bc7:512 (not a bench line)")
    ap.add_argument("--workload", default="c2", choices=["c2", "mips", "refine", "decode", "ranks"],
                    help="c2: the benchmark line; mips: batched mixed mip-chain workload; refine: gradient "
                         "endpoint refinement; decode: decode bandwidth (extra lines); ranks: the replica "
                         "plumbing on CPU (gloo)")
    ap.add_argument("--textures", type=int, default=64)
    ap.add_argument("--decode-size", type=int, default=8192)
    args = ap.parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_replicas(args.gpus, argv)
    world, rank, local = _dist()
    if args.workload == "ranks":
        ranks_selftest(args, world, rank)
    elif args.case:
        profile_case(args)
    elif args.workload == "mips":
        batched_mips_bench(args)
    elif args.workload == "refine":
        refine_bench(args)
    elif args.workload == "decode":
        decode_bench(args)
    elif args.impl == "reference":
        cpu_reference(args, world, rank)
    else:
        gpu_bench(args, world, rank, local)
    return 0


if __name__ == "__main__":
    sys.exit(main())
