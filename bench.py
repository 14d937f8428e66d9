"""Benchmark of the cloud-rendering hot path on B200.

Workload (one step = one frame): the neural form of the renderer (render type
MRPNN) on a 512^3 seeded Perlin-fBm cloud with its full mip pyramid, at
1920 x 1080, 1 primary sample per pixel, fp32 network (Xavier weights from
seed 1), extinction scale 64, albedo 0.99, g = 0.857, one seeded directional
light, camera at distance 2.5 with a 40 degree field of view. Synthetic
inputs; the volume is generated on the GPU before timing.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU runs are independent replicas (each rank renders its own frames;
no collective on the data path); `value` is the frames of all ranks divided by
the slowest rank's device time. `--impl reference` times the CPU
restatement of the reference path (the oracle, OpenMP on all host cores) on
a bounded sample of rows of the same frame, with the same weights, stencil
and tables; it loads no part of the library (the weights and the stencil come
from the oracle, the render request from internship_b200/scenes.py loaded as
a plain file). Both arms also report the delta-tracking baseline of the
sphere scene (128^3, 256 x 256, 64 spp) on the host cores.

Extra legs of the default run: the same frame with the texture sampler and
with the BF16 / FP8 tensor-core networks; the sphere scene's delta tracking on
the GPU (samples/s, density fetches/s, against the measured L2 read
bandwidth); an L2 / HBM read-bandwidth probe; batched serving; neural vs delta
tracking at matched RMSE against a 16384-spp FP64 image at 1920 x 1080; a
reduced training run (labels, training throughput, held-out error).
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "frames/s at 1080p, neural vs delta-tracking at matched RMSE vs 16k-spp oracle"
WIDTH, HEIGHT, RES = 1920, 1080, 512
FLOP_PER_PIXEL = 97072  # 48,536 MAC of the network per active pixel and albedo channel
WORKLOAD = ("neural (MRPNN) render 1920x1080, 1 spp, 512^3 Perlin-fBm cloud (6 oct, f0 4, lac 2, gain 0.5, "
            "thr 0.45, radial falloff), fp32 network, Xavier(seed 1) weights, reference stencil, alpha 64, "
            "albedo 0.99, g 0.857")


def config_dict():
    """The `config` of both arms' lines (identical by construction)."""
    return {"workload": WORKLOAD, "frame": "%dx%d" % (WIDTH, HEIGHT), "volume": "%d^3" % RES,
            "sampler": "exact fp32 trilinear", "network": "fp32",
            "l2": "flushed between steps (256 MiB write outside the timed events)"}


def load_scenes():
    """internship_b200/scenes.py as a plain module (no package import, so no
    library is loaded)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mr_scenes_plain", os.path.join(ROOT, "internship_b200", "scenes.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# the delta-tracking baseline scene: 128^3 sphere, 256 x 256, 64 spp
DT_W, DT_H, DT_SPP = 256, 256, 64


def cpu_delta_tracking():
    """The oracle's delta tracker (CalculateRadiance restated) on the sphere
    scene, OpenMP over rows on all host cores: the whole 256 x 256 x 64 image."""
    from oracle import orc
    sc = load_scenes()
    dens, p = sc.sphere_density(128), sc.make_params(DT_W, DT_H, DT_SPP, params_cls=orc.RenderParams)
    t0 = time.perf_counter()
    _, _, cnt = orc.render_pt(dens, float(dens.max()), p)
    dt = time.perf_counter() - t0
    n = DT_W * DT_H * DT_SPP
    return {"value": n / dt, "unit": "samples/s", "cores": orc.nthreads(), "kind": "port",
            "seconds": dt, "density_fetches_per_s": float(cnt[0]) / dt,
            "sample": "the whole sphere scene: 128^3, 256x256, 64 spp, 512 bounces (oracle, OpenMP)"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples every 50 ms during the timed legs."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q,
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference(args, rank):
    """CPU restatement (oracle) of the reference path on the host cores: the
    neural render of the benchmark frame, a bounded sample of rows per step,
    with the benchmark's weights, stencil and tables. Loads no part of the
    library."""
    if rank != 0:
        return
    from oracle import orc
    sc = load_scenes()
    threads = orc.nthreads()
    dens = orc.cloud(RES, 7)
    md, mips, _ = orc.build_mips(dens)
    p = sc.cloud_scene_params(WIDTH, HEIGHT, params_cls=orc.RenderParams)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    tr = orc.build_tr(mips, p.alpha, L)
    lut = orc.build_hglut(p.g, p.seed)
    w, st = orc.xavier_weights(1), orc.reference_stencil()
    rows_per_step = 16
    rows = np.linspace(0, HEIGHT - 1, rows_per_step * (args.steps + args.warmup)).astype(int)
    times = []
    for k in range(args.warmup + args.steps):
        sel = rows[k::args.warmup + args.steps]
        t0 = time.perf_counter()
        for r in sel:
            orc.render_neural(dens, md, mips, tr, lut, w, st, p, int(r), int(r) + 1)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    t = float(np.sum(times))
    frames = args.steps * rows_per_step / HEIGHT
    fps = frames / t
    line = {"metric": METRIC, "value": fps, "unit": "frames/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic", "config": config_dict(),
            "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": threads, "kind": "port",
                             "sample": "%d of %d rows per step, rows spread over the frame (host cores, OpenMP)"
                                       % (rows_per_step, HEIGHT)},
            "delta_tracking": cpu_delta_tracking(),
            "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


TRAINED = os.path.join(ROOT, "internship_b200", "data", "mrpnn_trained.npy")

# DRAM bytes (read + write) per unit from one ncu capture of each kernel on the
# 960x540 case of this frame (ncu --set full, one launch each): per active pixel
# for the gathers and networks (the fp32 network: k_simt_trunk + k_light_trunk +
# k_tc32_head + k_tc32_tail),
# per density fetch for the trace. A launch's traffic = this figure x the
# launch's units.
TRAFFIC_PER_UNIT = {"k_simt": 3377.8, "k_simt_trunk": 2103.4, "k_mlp_tc": 2456.3, "k_gather_fm_exact": 2463.2,
                    "k_gather_fm_texture": 2447.0, "k_nn_trace": 52.56}
# k_nn_trace: dram__bytes_read + write of one launch of the 1080p bench frame
# (759.9 MB for 14.46 M density fetches); the others at 960x540 per active pixel.
SIMT_KERNELS = ("k_simt_trunk + k_light_trunk + k_tc32_head + k_tc32_tail (fp32 network: CUDA-core trunks, "
                "tcgen05 head with fp32-accurate three-term TF32 products, CUDA-core tail)")
# The library's kernels of one fp32 / exact-sampler frame, in launch order
# (as an ncu launch list of this command shows them).
FP32_FRAME_KERNELS = ("k_sphere_h0", "k_nn_trace", "k_gather_fm", "k_simt_trunk", "k_light_trunk", "k_tc32_head",
                      "k_tc32_tail")
# algorithmic FLOPs per active pixel of the fp32 main-trunk kernel (blocks 0..7 and L81)
TRUNK_FLOP_PER_PIXEL = 32.9e3
# fp32 FMA rate of the CUDA cores (148 SMs x 128 lanes x 2 FLOP x 1.965 GHz), nominal
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def matched_rmse(v, p, sp, oracle_spp=16384, small=None):
    """Neural vs delta tracking at matched RMSE against an FP64-accumulated
    `oracle_spp` delta-tracking image of the same view.

    Errors are measured at the frame's own resolution (or at `small`, same
    camera) and converted into frames/s: delta tracking is unbiased, so its RMSE at s spp is c / sqrt(s) with c
    fitted over s = 1..64; the matched spp is s* = (c / RMSE_neural)^2 and the
    delta-tracking frame rate at matched RMSE is 1 / (s* t1), t1 = the measured
    time of one 1-spp 1080p delta-tracking frame. The neural form uses the
    network trained by internship_b200.train (BF16 tensor cores, texture
    sampler, one pass per frame)."""
    import torch
    import internship_b200 as mr
    from internship_b200 import _lib
    L = _lib.load()
    if not os.path.exists(TRAINED):
        return {"unavailable": "no trained weights at internship_b200/data/mrpnn_trained.npy"}
    w_tr = np.load(TRAINED)
    net = mr.Network(w_tr, mr.builtin_stencil())  # the shipped weights were trained on the reference stencil
    W, H = small if small else (p.width, p.height)
    q = _lib.RenderParams.from_buffer_copy(p)
    q.width, q.height = W, H
    npx = W * H * 3
    # oracle: FP64 sums over oracle_spp samples (seed 1000, independent of the measured images)
    s64 = torch.zeros(npx, device="cuda", dtype=torch.float64)
    q.render_type, q.seed, q.spp = _lib.RT_PT, 1000, 256
    torch.cuda.synchronize()
    t0 = time.time()
    for k in range(oracle_spp // 256):
        q.sample_offset = 256 * k
        _lib.check(L.mr_render_accumulate_f64(v.handle, C.byref(q), C.c_void_p(s64.data_ptr()), None, sp))
    torch.cuda.synchronize()
    t_oracle = time.time() - t0
    oracle = (s64 / oracle_spp).float()
    img = torch.empty(npx, device="cuda")

    def rmse(x):
        return float(torch.sqrt(torch.mean((x - oracle) ** 2)))

    # delta tracking at s spp (seed 2000)
    q.seed = 2000
    dt = {}
    for spp in (1, 4, 16, 64):
        q.spp, q.sample_offset = spp, 0
        _lib.check(L.mr_render(v.handle, None, C.byref(q), C.c_void_p(img.data_ptr()), sp))
        torch.cuda.synchronize()
        dt[spp] = rmse(img)
    c = float(np.exp(np.mean([np.log(e * np.sqrt(s)) for s, e in dt.items()])))
    # neural form, trained weights, one pass per frame; same LUT seed as the bench frames
    q.render_type, q.spp, q.seed = _lib.RT_MRPNN, 1, p.seed
    out = {}
    for name, prec, smp in (("fp32_exact", _lib.PREC_FP32, _lib.SAMPLER_EXACT),
                            ("bf16_exact", _lib.PREC_BF16, _lib.SAMPLER_EXACT),
                            ("bf16_texture", _lib.PREC_BF16, _lib.SAMPLER_TEXTURE),
                            ("fp8_exact", _lib.PREC_FP8, _lib.SAMPLER_EXACT)):
        q.precision, q.sampler = prec, smp
        errs, imgs = [], []
        for k in range(8):
            q.sample_offset = 50 + k
            _lib.check(L.mr_render(v.handle, net.handle, C.byref(q), C.c_void_p(img.data_ptr()), sp))
            torch.cuda.synchronize()
            errs.append(rmse(img))
            imgs.append(img.clone())
        out[name] = {"rmse_1pass": float(np.mean(errs)), "imgs": imgs}
    ref32 = torch.stack(out["fp32_exact"]["imgs"])
    for name in out:
        x = torch.stack(out[name].pop("imgs"))
        rel = torch.abs(x - ref32) / (torch.abs(ref32) + 1e-3)
        out[name]["max_rel_vs_fp32"] = float(rel.max())
        out[name]["rmse_vs_fp32"] = float(torch.sqrt(torch.mean((x - ref32) ** 2)))
    # 1-spp delta tracking at 1080p
    q.width, q.height = p.width, p.height
    q.render_type, q.spp, q.seed = _lib.RT_PT, 1, 3000
    full = torch.empty(p.width * p.height * 3, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(2):
        q.sample_offset = k
        _lib.check(L.mr_render(v.handle, None, C.byref(q), C.c_void_p(full.data_ptr()), sp))
    reps = 5
    e0.record()
    for k in range(reps):
        q.sample_offset = 10 + k
        _lib.check(L.mr_render(v.handle, None, C.byref(q), C.c_void_p(full.data_ptr()), sp))
    e1.record()
    torch.cuda.synchronize()
    t1 = e0.elapsed_time(e1) / reps / 1000.0
    net.close()
    e_nn = out["bf16_texture"]["rmse_1pass"]
    s_star = (c / e_nn) ** 2
    return {"oracle": {"spp": oracle_spp, "resolution": "%dx%d" % (W, H), "accumulation": "fp64",
                       "seconds": t_oracle},
            "dt_rmse_by_spp": {str(k): e for k, e in dt.items()}, "dt_rmse_coefficient": c,
            "neural": out, "matched_spp": s_star, "dt_1080p_ms_per_spp": 1000 * t1,
            "dt_1080p_samples_per_s": p.width * p.height / t1,
            "dt_fps_at_matched_rmse": 1.0 / (s_star * t1),
            "weights": "trained by internship_b200.train (config: 32 fBm clouds, 4096-spp FP64 labels)"}


BATCH_SIZES = [(256, 256), (512, 512), (1024, 576), (1280, 720), (1920, 1080)]


def batched_serving(replays=10, seed=11):
    """64 seeded fBm clouds (16 each of 64^3, 128^3, 256^3, 512^3), each seen
    from 4 random views at sizes drawn from 256x256 .. 1920x1080, BF16
    tensor-core network with the texture sampler, rendered as one batch per
    CUDA-graph replay with autotuned wave and block sizes. Reports aggregate
    pixels/s and the p50 / p99 latency of a batch frame (all 256 views)."""
    import torch
    import internship_b200 as mr
    from internship_b200 import _lib, scenes
    L = _lib.load()
    stream = torch.cuda.Stream()  # graph capture needs a stream other than the legacy default
    sp = C.c_void_p(stream.cuda_stream)
    torch.cuda.synchronize()
    rng = np.random.default_rng(seed)
    trained = os.path.exists(TRAINED)
    w = np.load(TRAINED) if trained else mr.xavier_weights(1)
    net = mr.Network(w, mr.builtin_stencil())
    vols, outs, frames = [], [], []
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    t0 = time.time()
    for c in range(64):
        res = (64, 128, 256, 512)[c // 16]
        with torch.cuda.stream(stream):
            dens = torch.empty(res ** 3, device="cuda")
        scenes.generate_cloud_device(res, 2000 + c, dens.data_ptr(), sp)
        v = mr.VolumeRender(res)
        _lib.check(L.mr_volume_set_data_device(v.handle, C.c_void_p(dens.data_ptr()), dens.numel(), sp))
        _lib.check(L.mr_volume_update(v.handle, sp))
        del dens
        vols.append(v)
        light = int(rng.integers(1 << 30))
        for k in range(4):
            W, H = BATCH_SIZES[int(rng.integers(len(BATCH_SIZES)))]
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            p = scenes.make_params(W, H, 1, rt=_lib.RT_MRPNN, precision=_lib.PREC_BF16,
                                   sampler=_lib.SAMPLER_TEXTURE, light_seed=light)
            ori, up, right = scenes.camera_vectors(d * 2.5, 40.0)
            p.ori, p.up, p.right = _lib.f3(ori), _lib.f3(up), _lib.f3(right)
            with torch.cuda.stream(stream):
                o = torch.empty(W * H * 3, device="cuda")
            outs.append(o)
            frames.append((W, H))
            _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), C.c_void_p(o.data_ptr())))
    _lib.check(L.mr_batch_prepare(b, net.handle, 0, sp))
    t_setup = time.time() - t0
    wave, tb, gb = C.c_int64(), C.c_int32(), C.c_int32()
    _lib.check(L.mr_batch_autotune(b, net.handle, C.byref(wave), C.byref(tb), C.byref(gb), sp))
    _lib.check(L.mr_batch_set_timing(b, 1))  # per-frame completion events inside the graph
    _lib.check(L.mr_batch_capture(b, net.handle, sp))
    for _ in range(2):
        _lib.check(L.mr_batch_launch(b, sp))
    torch.cuda.synchronize()
    lat, frame_ms, frame_err = [], [], None
    ft = np.zeros(len(frames), np.float32)
    for _ in range(replays):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(L.mr_batch_launch(b, sp))
        e1.record(stream)
        torch.cuda.synchronize()
        lat.append(e0.elapsed_time(e1))
        if frame_ms is not None:
            rc = L.mr_batch_frame_times(b, ft.ctypes.data, len(frames))
            if rc == _lib.MR_OK:
                frame_ms.append(ft.copy())
            else:  # per-frame times unavailable: the batch latency stands alone
                frame_err, frame_ms = L.mr_last_error().decode(), None
    cnt = (C.c_uint64 * 4)()
    _lib.check(L.mr_batch_counters(b, cnt))
    total_px = sum(W * H for W, H in frames)
    L.mr_batch_destroy(b)
    for v in vols:
        v.close()
    net.close()
    lat = np.array(lat)
    return {"workload": "64 fBm clouds (16 x 64^3/128^3/256^3/512^3) x 4 views, sizes 256^2..1920x1080, "
                        "BF16 network, texture sampler, trained weights",
            "frames_per_batch": len(frames), "pixels_per_batch": total_px,
            "pixels_per_s": total_px / (float(np.mean(lat)) / 1000.0),
            "frames_per_s": len(frames) / (float(np.mean(lat)) / 1000.0),
            "batch_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                 "mean": float(np.mean(lat))},
            "frame_latency_ms": {"p50": float(np.percentile(np.concatenate(frame_ms), 50)),
                                 "p99": float(np.percentile(np.concatenate(frame_ms), 99)),
                                 "definition": "from the batch frame's start to the completion of the wave holding "
                                               "the frame's last pixel (device-timer stamps in the captured graph)"}
            if frame_ms else {"unavailable": frame_err},
            "autotuned": {"wave_pixels": int(wave.value), "trace_block": int(tb.value), "gather_block": int(gb.value)},
            "replays": replays, "graph": "one CUDA graph per batch frame", "setup_s": t_setup}


def memory_probe():
    """Read bandwidth of L2 (a 24 MiB buffer, resident after the first pass)
    and of HBM (a 4 GiB buffer) through mr_stream_read_probe: 16-byte loads
    that bypass L1, timed with events on the launching stream."""
    import torch
    from internship_b200 import _lib
    L = _lib.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    sink = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = {}
    for name, mib, passes in (("l2", 24, 400), ("hbm", 4096, 3)):
        buf = torch.ones(mib * 1024 * 1024 // 4, device="cuda")
        nbytes = buf.numel() * 4
        for _ in range(2):
            _lib.check(L.mr_stream_read_probe(C.c_void_p(buf.data_ptr()), nbytes, passes, C.c_void_p(sink.data_ptr()),
                                              sp))
        best = 0.0
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.check(L.mr_stream_read_probe(C.c_void_p(buf.data_ptr()), nbytes, passes,
                                              C.c_void_p(sink.data_ptr()), sp))
            e1.record(stream)
            torch.cuda.synchronize()
            best = max(best, nbytes * passes / (e0.elapsed_time(e1) / 1e3) / 1e9)
        out[name + "_read_gbs"] = best
        del buf
        torch.cuda.empty_cache()  # the 4 GiB buffer leaves the device, not just the allocator's cache
    out["method"] = "mr_stream_read_probe: ld.global.cg 16-byte loads, 24 MiB x 400 passes (L2), 4 GiB x 3 (HBM); best of 5"
    return out


def gpu_delta_tracking(l2_gbs, steps=10):
    """Delta tracking of the sphere scene on the GPU (128^3, 256 x 256, 64 spp,
    512 bounces, unit light): samples/s and density fetches/s, the fetch
    stream's algorithmic bytes (32 B per trilinear fetch) against the
    measured L2 read bandwidth (the 8 MiB grid stays in L2)."""
    import torch
    import internship_b200 as mr
    from internship_b200 import _lib, scenes
    L = _lib.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    dens, p = scenes.sphere_scene(DT_W, DT_H, DT_SPP)
    v = mr.VolumeRender(128)
    v.SetDatas(dens)
    v.Update()
    out = torch.empty(DT_W * DT_H * 3, device="cuda")
    for k in range(3):
        p.sample_offset = 1000 * k
        _lib.check(L.mr_render(v.handle, None, C.byref(p), C.c_void_p(out.data_ptr()), sp))
    torch.cuda.synchronize()
    ms, fetches = 0.0, 0
    cnt = (C.c_uint64 * 4)()
    for k in range(steps):
        p.sample_offset = 10000 + DT_SPP * k
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(L.mr_render(v.handle, None, C.byref(p), C.c_void_p(out.data_ptr()), sp))
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        _lib.check(L.mr_volume_counters(v.handle, cnt))
        fetches += int(cnt[0])
    v.close()
    sec = ms / 1e3
    n = steps * DT_W * DT_H * DT_SPP
    ach = fetches * 32.0 / sec / 1e9
    return {"workload": "delta tracking, 128^3 sphere (alpha 64, albedo 0.99, g 0.857), 256x256, 64 spp, "
                        "512 bounces", "kernel": "k_delta_track",
            "samples_per_s": n / sec, "density_fetches_per_s": fetches / sec, "ms_per_frame": ms / steps,
            "frames": steps,
            "roofline": {"bound": "l2", "achieved": ach, "peak": l2_gbs, "unit": "GB/s", "frac": ach / l2_gbs,
                         "peak_source": "measured in this run (mr_stream_read_probe, 24 MiB)",
                         "algorithmic_bytes": "32 B per trilinear density fetch"}}


def denoise_leg(hbm_gbs, steps=10, W=1920, H=1080):
    """The histogram denoiser alone (mr_denoise: Compare-weighted 11 x 11
    filter, ACES, pack) on a 1080p accumulation whose every pixel is above the
    variance threshold (the filter runs everywhere). Algorithmic bytes per
    pixel: the 33-float histogram and 3-float colour read once, the packed
    pixel written: 148 B. The 307 MB of inputs exceed L2."""
    import torch
    from internship_b200 import _lib
    L = _lib.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(3)
    n = W * H
    acc = torch.rand(n * 3, device="cuda", generator=g) * 2.0
    hist = torch.zeros(n, 33, device="cuda")
    hist[:, :30] = torch.randint(0, 4, (n, 30), device="cuda", generator=g).float()
    hist[:, 30] = 16.0
    hist[:, 31] = 0.6  # mean of l^2
    hist[:, 32] = 0.5  # mean of l: variance 0.35 > 0.01
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    it = _lib.Interactive()
    it.frame_index, it.tone, it.denoise, it.checkerboard, it.exposure = 16, 2, 1, 0, 1.0

    def run():
        _lib.check(L.mr_denoise(C.c_void_p(acc.data_ptr()), C.c_void_p(hist.data_ptr()), C.c_void_p(out.data_ptr()),
                                W, H, C.byref(it), sp))
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = float(np.mean(ms))
    ach = n * 148.0 / (t / 1e3) / 1e9
    return {"workload": "mr_denoise at %dx%d, ACES, filter active on every pixel" % (W, H), "kernel": "k_denoise",
            "ms": t, "pixels_per_s": n / (t / 1e3),
            "compare_bin_terms_per_s": n * 121 * 30 / (t / 1e3),
            "bound": "instruction issue and the XU pipe (121 x 30 Compare bin terms per pixel, one approximate "
                     "reciprocal each), not HBM",
            "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm_gbs, "unit": "GB/s", "frac": ach / hbm_gbs,
                         "algorithmic_bytes": "148 B per pixel (histogram 132 B + colour 12 B read, 4 B written)"}}


def training_leg(configs=8, samples=400_000, spp=1024, epochs=20):
    """Reduced configuration-4 run of the learned part: labels from the
    project's delta tracker on seeded fBm clouds (FP64 sums), training with
    the hand-written kernels (BF16 tensor-core head, FP32 master weights and
    Adam), held-out error with and without the network."""
    from internship_b200 import train
    _, rep = train.run(configs=configs, samples=samples, spp=spp, bounces=512, epochs=epochs, batch=65536, lr=1e-3,
                       precision="bf16")
    rep["workload"] = ("%d seeded fBm clouds (128^3 / 256^3 / 512^3), alpha 16-256, albedo 0.9-1.0, g 0.7-0.9, "
                       "%d rows, %d spp per label, %d epochs (configuration 4 reduced: 32 clouds, 5 M rows, "
                       "4096 spp)" % (configs, samples, spp, epochs))
    return rep


def cpu_baseline_sample(v, dens_dev, p, w, st):
    """Bounded sample of the same frame on the oracle (all host cores)."""
    from internship_b200 import _lib
    from oracle import orc
    dens = dens_dev.cpu().numpy()
    mips = np.concatenate([v.read(_lib.READ_MIP, k) for k in range(9)])
    tr = np.concatenate([v.read(_lib.READ_TR, k) for k in range(8)])
    lut = v.read(_lib.READ_HGLUT)
    rows = np.linspace(0, HEIGHT - 1, 24).astype(int)
    t0 = time.perf_counter()
    for r in rows:
        orc.render_neural(dens, v.max_density, mips, tr, lut, w, st, p, int(r), int(r) + 1)
    dt = time.perf_counter() - t0
    fps = (len(rows) / HEIGHT) / dt
    return {"value": fps, "unit": "frames/s", "cores": orc.nthreads(), "kind": "port",
            "sample": "%d of %d rows of one frame (oracle, OpenMP)" % (len(rows), HEIGHT)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-rmse", action="store_true", help="skip the matched-RMSE comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-serving measurement")
    ap.add_argument("--no-train", action="store_true", help="skip the reduced training run")
    ap.add_argument("--no-probe", action="store_true",
                    help="skip the L2 / HBM read probe (its 4 GiB buffer) and the delta-tracking leg: profiler runs")
    ap.add_argument("--frame", default=None,
                    help="WxH instead of 1920x1080: a smaller case for profiler captures, not a bench line")
    ap.add_argument("--denoise-only", default=None, metavar="WxH",
                    help="run only the histogram-denoiser leg at WxH and print its record: profiler runs")
    args = ap.parse_args()
    if args.frame:
        global WIDTH, HEIGHT
        WIDTH, HEIGHT = (int(x) for x in args.frame.lower().split("x"))
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        run_reference(args, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    torch.cuda.set_device(local)
    if args.denoise_only:
        dw, dh = (int(x) for x in args.denoise_only.lower().split("x"))
        print(json.dumps(denoise_leg(peaks()[0], steps=args.steps, W=dw, H=dh)), flush=True)
        return
    import internship_b200 as mr
    from internship_b200 import _lib, replicas, scenes
    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    sp = C.c_void_p(stream)

    # -- inputs: cloud generated on the device, tables built, network uploaded
    dens = torch.empty(RES ** 3, device="cuda", dtype=torch.float32)
    scenes.generate_cloud_device(RES, 7, dens.data_ptr(), sp)
    v = mr.VolumeRender(RES)
    _lib.check(L.mr_volume_set_data_device(v.handle, C.c_void_p(dens.data_ptr()), dens.numel(), sp))
    _lib.check(L.mr_volume_update(v.handle, sp))
    md = C.c_float()
    _lib.check(L.mr_volume_max_density(v.handle, C.byref(md)))
    v.max_density = md.value
    w, st = mr.xavier_weights(1), mr.builtin_stencil()
    v.SetWeights(w, st)
    net = v.network.handle
    p = scenes.cloud_scene_params(WIDTH, HEIGHT, seed=replicas.frame_seed(rank))
    out = torch.empty(WIDTH * HEIGHT * 3, device="cuda", dtype=torch.float32)
    flush = torch.empty(256 * 1024 * 1024 // 4, device="cuda", dtype=torch.float32)

    def render(step):
        p.sample_offset = step
        _lib.check(L.mr_render(v.handle, net, C.byref(p), C.c_void_p(out.data_ptr()), sp))

    def leg(precision, sampler, base):
        """Time args.steps frames (L2 flushed between steps, outside the events)
        with per-stage events inside the library; returns the max-over-ranks
        device time, per-stage means and the last frame's counters."""
        p.precision, p.sampler = precision, sampler
        for k in range(args.warmup):
            render(base + k)
        torch.cuda.synchronize()
        L.mr_volume_stage_times(v.handle, (C.c_double * 8)(), (C.c_int32 * 8)(), 8)  # reset
        _lib.check(L.mr_volume_set_timing(v.handle, 1))
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record()
            render(base + 100 + k)
            evs[k][1].record()
        torch.cuda.synchronize()
        ms = float(sum(a.elapsed_time(b) for a, b in evs))
        st_ms = (C.c_double * 8)()
        st_n = (C.c_int32 * 8)()
        _lib.check(L.mr_volume_stage_times(v.handle, st_ms, st_n, 8))
        _lib.check(L.mr_volume_set_timing(v.handle, 0))
        _lib.check(L.mr_network_check(net, 1))
        cnt = (C.c_uint64 * 4)()
        _lib.check(L.mr_volume_counters(v.handle, cnt))
        if dist is not None:
            ms = replicas.slowest_ms(ms, dist, "cuda")
            dist.barrier()
        per = [st_ms[i] / max(1, st_n[i]) for i in range(8)]
        return {"ms": ms, "stage": per, "launches": int(sum(st_n[i] for i in range(8))),
                "active": int(cnt[3]), "fetches": int(cnt[0])}

    # fp32 network, exact sampler: the headline configuration
    # clocks sampled over all the timed legs below (nvidia-smi needs a moment to start)
    clocks = ClockSampler(torch.cuda.current_device())
    time.sleep(0.5)
    head = leg(_lib.PREC_FP32, _lib.SAMPLER_EXACT, 0)
    ms, active, fetches = head["ms"], head["active"], head["fetches"]
    fps = replicas.throughput(args.steps, world, ms)
    # the same frames with texture-unit sampling and with the BF16 tensor-core network
    legs = {"fp32_texture": leg(_lib.PREC_FP32, _lib.SAMPLER_TEXTURE, 1000),
            "bf16_exact": leg(_lib.PREC_BF16, _lib.SAMPLER_EXACT, 2000),
            "bf16_texture": leg(_lib.PREC_BF16, _lib.SAMPLER_TEXTURE, 3000),
            "fp8_texture": leg(_lib.PREC_FP8, _lib.SAMPLER_TEXTURE, 4000)}
    p.precision, p.sampler = _lib.PREC_FP32, _lib.SAMPLER_EXACT
    clk = clocks.stop()

    # -- end to end through the public API, frames delivered to pinned host
    # memory: mr_render_host_async renders frame k+1 while frame k's copy runs
    # (two device frames owned by the volume). Host wall clock from an idle
    # device to the last frame in host memory.
    hosts = [torch.empty(WIDTH * HEIGHT * 3, dtype=torch.float32, pin_memory=True) for _ in range(2)]
    ticket = C.c_int64()

    def render_to_host(step):
        p.sample_offset = step
        _lib.check(L.mr_render_host_async(v.handle, net, C.byref(p), C.c_void_p(hosts[step % 2].data_ptr()), sp,
                                          C.byref(ticket)))

    for k in range(args.warmup):
        render_to_host(4900 + k)
    _lib.check(L.mr_render_host_wait(v.handle, -1, 60000))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        render_to_host(5000 + k)
    _lib.check(L.mr_render_host_wait(v.handle, -1, 60000))
    e2e_ms = (time.perf_counter() - t0) * 1e3
    e2e_ms = replicas.slowest_ms(e2e_ms, dist, "cuda")
    e2e_fps = replicas.throughput(args.steps, world, e2e_ms)
    # the same without overlap: each frame rendered, then copied, on one stream
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        render(5100 + k)
        hosts[0].copy_(out, non_blocking=True)
    torch.cuda.synchronize()
    serial_ms = replicas.slowest_ms((time.perf_counter() - t0) * 1e3, dist, "cuda")
    serial_fps = replicas.throughput(args.steps, world, serial_ms)

    hbm, bf16, src = peaks()
    probe = memory_probe() if not args.no_probe else {"l2_read_gbs": float("nan"), "skipped": True}
    l2 = probe["l2_read_gbs"]
    trace_ms, gather_ms, mlp_ms32 = head["stage"][1], head["stage"][2], head["stage"][6]
    # algorithmic bytes: trace = density fetches x 32 B (8 fp32 texels);
    # gather = 192 + 192 trilinear fetches x 32 B + 383 bilinear x 16 B + the
    # 581 fp32 descriptor values written, per active pixel.
    trace_bytes = fetches * 32.0
    gather_bytes = active * (384 * 32 + 383 * 16 + 581 * 4)
    stages = {
        "nn_trace": {"bound": "hbm", "kernel": "k_nn_trace", "ms": trace_ms,
                     "achieved": trace_bytes / (trace_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s"},
        "nn_gather": {"bound": "l2", "kernel": "k_gather_fm<kSampGather> (exact sampler, texture gathers)",
                      "ms": gather_ms, "achieved": gather_bytes / (gather_ms / 1e3) / 1e9, "peak": l2, "unit": "GB/s"},
        "nn_network": {"bound": "tensor", "kernel": SIMT_KERNELS, "ms": mlp_ms32,
                       "achieved": FLOP_PER_PIXEL * active / (mlp_ms32 / 1e3) / 1e12, "peak": bf16,
                       "unit": "TFLOP/s"},
    }
    for s_ in stages.values():
        s_["frac"] = s_["achieved"] / s_["peak"]
        s_["peak_source"] = src
    stages["nn_gather"]["peak_source"] = "measured in this run (L2 read probe, 24 MiB)"
    stages["nn_trace"]["traffic"] = TRAFFIC_PER_UNIT["k_nn_trace"] * fetches
    stages["nn_gather"]["traffic"] = TRAFFIC_PER_UNIT["k_gather_fm_exact"] * active
    stages["nn_network"]["traffic"] = TRAFFIC_PER_UNIT["k_simt"] * active
    stages["nn_network"]["fp32_fma_peak"] = FP32_PEAK_TFLOPS
    stages["nn_network"]["frac_of_fp32_fma_peak"] = stages["nn_network"]["achieved"] / FP32_PEAK_TFLOPS
    for s_ in stages.values():
        s_["traffic_source"] = "ncu dram__bytes_read+write per unit at 960x540, scaled by this launch's units"
    stages["nn_trace"]["traffic_source"] = ("ncu dram__bytes_read+write of one 1080p launch (52.56 B per fetch), "
                                            "scaled by this launch's fetches")
    # the dominant single kernel of the frame: the trace, the gather, or the
    # largest of the network's four kernels (the main trunk, timed on its own
    # as library stage 7)
    trunk_ms = head["stage"][7]
    kernels = {"k_nn_trace": dict(stages["nn_trace"], stage="nn_trace"),
               "k_gather_fm": dict(stages["nn_gather"], stage="nn_gather"),
               "k_simt_trunk": {"bound": "fp32", "kernel": "k_simt_trunk (fp32 main trunk on the CUDA cores)",
                                "ms": trunk_ms,
                                "achieved": TRUNK_FLOP_PER_PIXEL * active / (trunk_ms / 1e3) / 1e12,
                                "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s",
                                "peak_source": "nominal fp32 FMA rate (148 SMs x 128 lanes x 2 x 1.965 GHz)",
                                "stage": "nn_network"}}
    kernels["k_simt_trunk"]["frac"] = kernels["k_simt_trunk"]["achieved"] / FP32_PEAK_TFLOPS
    kernels["k_simt_trunk"]["traffic"] = TRAFFIC_PER_UNIT["k_simt_trunk"] * active
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    roofline = kernels[dom]
    stages["nn_network"]["largest_kernel"] = {"kernel": "k_simt_trunk", "ms": trunk_ms}
    variants = {}
    for name, lg in legs.items():
        g_ms, m_ms = lg["stage"][2], lg["stage"][6]
        tc = not name.startswith("fp32")
        tf = FLOP_PER_PIXEL * lg["active"] / (m_ms / 1e3) / 1e12
        variants[name] = {
            "value": replicas.throughput(args.steps, world, lg["ms"]), "unit": "frames/s",
            "ms_per_step": lg["ms"] / args.steps,
            "stages_ms_per_step": {"nn_trace": lg["stage"][1], "nn_gather": g_ms, "nn_network": m_ms},
            "gather": {"bound": "l2", "achieved": lg["active"] * (384 * 32 + 383 * 16 + 581 * 4) / (g_ms / 1e3) / 1e9,
                       "peak": l2, "unit": "GB/s"},
            "network": {"bound": "tensor",
                        "kernel": ("k_mlp_tc (tcgen05 %s network)" % ("E4M3" if name.startswith("fp8") else "BF16"))
                        if tc else SIMT_KERNELS,
                        "achieved": tf, "peak": bf16, "unit": "TFLOP/s", "frac": tf / bf16, "peak_source": src,
                        "traffic": TRAFFIC_PER_UNIT["k_mlp_tc" if tc else "k_simt"] * lg["active"]},
        }
    line = {"metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": config_dict(),
            "parallelism": "replicas" if world > 1 else "single GPU",
            "e2e": {"value": e2e_fps, "unit": "frames/s", "h2d_bytes_per_step": C.sizeof(_lib.RenderParams),
                    "d2h_bytes_per_step": WIDTH * HEIGHT * 3 * 4,
                    "api": "mr_render_host_async (copy of frame k overlaps the render of frame k+1)",
                    "clock": "host wall clock to the last frame in pinned host memory",
                    "serial_value": serial_fps},
            "gpu_launches": args.steps * len(FP32_FRAME_KERNELS),
            "gpu_kernels_per_step": list(FP32_FRAME_KERNELS),
            "roofline": roofline, "clocks": clk,
            "stage_rooflines": stages,
            "active_pixels_per_frame": active,
            "density_fetches_per_frame": fetches,
            "variants": variants,
            "memory_probe": probe}
    if world == 1 and not args.no_probe:
        line["delta_tracking"] = gpu_delta_tracking(l2)
    if world == 1:
        line["denoise"] = denoise_leg(hbm)
    if not args.no_batch and world == 1:
        line["batched"] = batched_serving()
    if not args.no_rmse:
        m = matched_rmse(v, p, sp)
        if "matched_spp" in m:
            nn_fps = variants["bf16_texture"]["value"] / world
            m["neural_fps"] = nn_fps
            m["neural_over_dt_at_matched_rmse"] = nn_fps / m["dt_fps_at_matched_rmse"]
        line["matched_rmse"] = m
    if not args.no_train and world == 1:
        line["training"] = training_leg()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(v, dens, p, w, st)
        line["cpu_baseline"]["delta_tracking"] = cpu_delta_tracking()
    if rank == 0:
        print(json.dumps(line), flush=True)
    v.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
