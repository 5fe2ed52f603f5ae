"""Benchmark of the spectral shallow-water hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--quick]

Headline workload (one "step"), run in the mixed-precision form (Legendre
stage on tcgen05 kind::i8, integer split with exact int32 sums) with the FP64
form (Legendre stage on the FP64 tensor cores, mma.sync m8n8k4 f64) measured
beside it: the
transform-throughput configuration,
T255 on the 384 x 768 Gauss grid, 64 scalar fields plus 32 vorticity/divergence
pairs, inverse and forward transform of every field.  Metric: SHT GFLOP/s with
the algorithmic flop count 2*nlm*nlat per field per direction per Legendre
contraction (384 contractions) plus 2.5*nphi*log2(nphi)*nlat per field FFT
(256 field-FFTs): 11.51 GFLOP per step.

Inputs are synthetic (seeded complex N(0,1) spectra scaled by (l+1)^-1.5,
Im = 0 at m = 0) and larger than L2 (>= 270 MB per step), so no L2 flush is
needed between steps.  Also reported (not the headline): the FP64 form of the
same step, the per-field relative L2 of the mixed form against the FP64 path,
the Legendre stages alone (64 fields, and 1-8 fields as in the RK4 steps),
nonlinear RK4 steps/s at T255 (advective and vorticity-divergence forms) and
T63 (plain-method configuration) in both forms, REXI steps/s at T127 (M =
256, 535 poles; FP64 with stored factors, and the mixed form), the 256-member
uneven ensemble and T1023, each with its relative L2 against the FP64 form.

End to end (`e2e`): the same step through the public transform calls with
the input spectra in pinned host memory and the output spectra copied back to
pinned host memory every step (67 MB each way).  The reported figure runs the
steps pipelined (upload, compute and download streams; two device buffer
sets, so step k + 1's upload and step k - 1's download overlap step k's
transforms); `ms_per_step_serial` is the same steps one after another.

--impl reference times the CPU restatement of the same algorithm (the oracle;
the reference's SHTNS/FFTW/LAPACK build is unavailable on this machine) on the
host cores, on a bounded sample of the same workload.

Multi-GPU: the transform batch is independent per field, so N ranks each run
the full per-GPU workload (weak scaling, no collective in the data path).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L_CFG1 = 255
N_SCALAR = 64
N_PAIRS = 32
METRIC = "SWE steps/s & SHT GFLOP/s at T255/T127 REXI: mixed vs FP64-GPU at relL2<=1e-6"
# DRAM bytes (read + write) of one int8 Legendre analysis of 64 fields at T255
# (k_i8b_prep_ana<32> then k_legendre_i8b<AnaI8<32>>), from one ncu capture of
# the two launches (dram__bytes_read.sum + dram__bytes_write.sum of each):
# (101.38 + 17.54) + (88.50 + 6.63) MB
TRAFFIC_ANA64 = (101.38 + 17.54 + 88.50 + 6.63) * 1e6


def ana64_bytes(L=L_CFG1, nlat=384, nfields=N_SCALAR):
    """Algorithmic bytes of one Legendre analysis of nfields fields: the Fourier
    input read once, the int8 digit table of P_l^m w_j read once (4 bytes per
    (l, m, northern latitude)), the spectra written once."""
    nlm = (L + 1) * (L + 2) // 2
    return nfields * (L + 1) * nlat * 16 + nlm * (nlat // 2) * 4 + nfields * nlm * 16


def cfg1_flops(L=L_CFG1, nlat=384, nphi=768):
    nlm = (L + 1) * (L + 2) // 2
    per_contraction = 2.0 * nlm * nlat
    n_contr = N_SCALAR * 2 + N_PAIRS * 4 * 2
    fft_per_field = 2.5 * nphi * math.log2(nphi) * nlat
    n_fft = N_SCALAR * 2 + N_PAIRS * 2 * 2
    return per_contraction * n_contr, fft_per_field * n_fft, per_contraction


def random_spec(L, n, seed, zero_mean=False):
    """complex N(0,1) * (l+1)^-1.5, Im = 0 at m = 0; zero_mean drops the (0,0)
    coefficient (vorticity and divergence have no global mean)."""
    rng = np.random.default_rng(seed)
    nlm = (L + 1) * (L + 2) // 2
    ls = np.concatenate([np.arange(m, L + 1) for m in range(L + 1)])
    x = (rng.standard_normal((n, nlm)) + 1j * rng.standard_normal((n, nlm))) * (ls + 1.0) ** -1.5
    x[:, : L + 1] = x[:, : L + 1].real
    if zero_mean:
        x[:, 0] = 0
    return x


class ClockSampler:
    """SM clock and throttle reasons sampled DURING the timed region.

    NVML (nvidia-ml-py) is polled every ~2 ms from a host thread, so even a
    timed region of a few tens of milliseconds gets samples; nvidia-smi
    (100 ms interval) is the fallback where NVML cannot be loaded."""

    # NVML clocks-event-reason bits by their pynvml names
    REASON_NAMES = (("nvmlClocksEventReasonHwSlowdown", "hw_slowdown"),
                    ("nvmlClocksEventReasonHwThermalSlowdown", "hw_thermal_slowdown"),
                    ("nvmlClocksEventReasonHwPowerBrakeSlowdown", "hw_power_brake_slowdown"),
                    ("nvmlClocksEventReasonSwThermalSlowdown", "sw_thermal_slowdown"),
                    ("nvmlClocksEventReasonSwPowerCap", "sw_power_cap"))

    def __init__(self, index=0, period_s=0.002):
        self.index = index
        self.period = period_s
        self.samples = []  # (sm_mhz, max_mhz, [reasons])
        self.proc = None
        self.nvml = None
        self._stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.dev = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.dev, pynvml.NVML_CLOCK_SM))
            self.bits = [(int(getattr(pynvml, a)), n) for a, n in self.REASON_NAMES if hasattr(pynvml, a)]
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _poll(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.dev, nv.NVML_CLOCK_SM))
                bits = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.dev))
                self.samples.append((mhz, self.max_mhz, [n for b, n in self.bits if bits & b]))
            except Exception:
                return
            time.sleep(self.period)

    def _read(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            try:
                self.samples.append((float(f[0]), float(f[1]),
                                     [names[k] for k in range(4) if len(f) > 3 + k and f[3 + k] == "Active"]))
            except ValueError:
                pass

    def __exit__(self, *a):
        self._stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=2)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [x[0] for x in self.samples]
        reasons = sorted({r for x in self.samples for r in x[2]})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(x[1] for x in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ------------------------------------------------------------------ our arm
def _cfg1_inputs(dev, rank):
    import torch

    spec = torch.from_numpy(random_spec(L_CFG1, N_SCALAR, 1 + rank)).to(dev)
    vort = torch.from_numpy(random_spec(L_CFG1, N_PAIRS, 1001 + rank, zero_mean=True)).to(dev)
    div = torch.from_numpy(random_spec(L_CFG1, N_PAIRS, 2001 + rank, zero_mean=True)).to(dev)
    return spec, vort, div


class Cfg1:
    """One step of the transform-throughput configuration on one handle:
    synthesis + analysis of the scalar fields, vector synthesis + analysis of
    the vorticity/divergence pairs.  Kernel launches of the mixed form: scalar
    synthesis 3 (B preparation, int8 contraction, ring FFT) and analysis 3;
    vector synthesis 7 (degree-(L+1) spectra, B preparation, contraction, the
    FP64 orders m = 0, 1, the 1/cos scaling, two ring FFTs) and analysis 6
    (two ring FFTs, B preparation, contraction, FP64 m = 0, 1, recurrences)."""

    LAUNCHES = 3 + 3 + 7 + 6

    def __init__(self, prec, dev, spec, vort, div):
        import torch

        from sph_swe_b200.sph import Sph

        self.s = Sph(L_CFG1, precision=prec)
        assert (self.s.nlat, self.s.nphi) == (384, 768)
        # the autotuner picks the kernel variants for the step's batches (untimed
        # set-up): Legendre 64 fields (scalars; the 32 pairs' U, V), rings 64 / 32
        for b in sorted({N_SCALAR, 2 * N_PAIRS, N_PAIRS}):
            self.s.autotune(b)
        self.spec, self.vort, self.div = spec, vort, div
        self.grid = torch.empty(N_SCALAR, self.s.nphi, self.s.nlat, dtype=torch.float64, device=dev)
        self.spec_out = torch.empty_like(spec)
        self.u = self.v = self.z = self.d = None

    def step(self):
        s = self.s
        s.SH_to_spat(self.spec, out=self.grid)
        s.spat_to_SH(self.grid, out=self.spec_out)
        self.u, self.v = s.vec_SH_to_spat(self.vort, self.div)
        self.z, self.d = s.vec_spat_to_SH(self.u, self.v)

    def sync_ok(self):
        from sph_swe_b200 import capi

        capi.check(capi.lib().sph_sync(self.s.h, None))


def _time(fn, steps, st):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _e2e_pipelined(sph, h_spec, h_vort, h_div, o_spec, o_vort, o_div, steps, dev):
    """Milliseconds per step of config 1 end to end with host buffers, the
    copies of neighbouring steps overlapping the compute (see the caller)."""
    import torch

    s_in, s_cmp, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    sets = []
    for _ in range(2):
        b = {"spec": torch.empty(h_spec.shape, dtype=h_spec.dtype, device=dev),
             "vort": torch.empty(h_vort.shape, dtype=h_vort.dtype, device=dev),
             "div": torch.empty(h_div.shape, dtype=h_div.dtype, device=dev)}
        b["grid"] = torch.empty(N_SCALAR, sph.nphi, sph.nlat, dtype=torch.float64, device=dev)
        b["spec_out"] = torch.empty_like(b["spec"])
        b["u"] = torch.empty(N_PAIRS, sph.nphi, sph.nlat, dtype=torch.float64, device=dev)
        b["v"] = torch.empty_like(b["u"])
        b["z"] = torch.empty_like(b["vort"])
        b["d"] = torch.empty_like(b["div"])
        sets.append(b)
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_cmp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def run(n):
        for k in range(n):
            i = k % 2
            b = sets[i]
            with torch.cuda.stream(s_in):
                if k >= 2:
                    s_in.wait_event(ev_cmp[i])  # step k - 2 has consumed this set's inputs
                b["spec"].copy_(h_spec, non_blocking=True)
                b["vort"].copy_(h_vort, non_blocking=True)
                b["div"].copy_(h_div, non_blocking=True)
                ev_in[i].record(s_in)
            with torch.cuda.stream(s_cmp):
                s_cmp.wait_event(ev_in[i])
                if k >= 2:
                    s_cmp.wait_event(ev_out[i])  # step k - 2's results have left this set
                sph.SH_to_spat(b["spec"], out=b["grid"])
                sph.spat_to_SH(b["grid"], out=b["spec_out"])
                sph.vec_SH_to_spat(b["vort"], b["div"], out=(b["u"], b["v"]))
                sph.vec_spat_to_SH(b["u"], b["v"], out=(b["z"], b["d"]))
                ev_cmp[i].record(s_cmp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_cmp[i])
                o_spec.copy_(b["spec_out"], non_blocking=True)
                o_vort.copy_(b["z"], non_blocking=True)
                o_div.copy_(b["d"], non_blocking=True)
                ev_out[i].record(s_out)

    run(3)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    run(steps)
    s_out.wait_stream(s_in)
    s_out.wait_stream(s_cmp)
    e1.record(s_out)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    del sets
    return ms


def _max_over_ranks(ms, world, dev):
    """the slowest rank's time (NCCL on the device, or gloo on the host)"""
    import torch

    if world > 1:
        d = dev if torch.distributed.get_backend() == "nccl" else torch.device("cpu")
        t = torch.tensor([ms], device=d, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def _per_field_rel(a, b):
    import torch

    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    r = torch.linalg.vector_norm(a - b, dim=1) / torch.linalg.vector_norm(b, dim=1)
    return {"max": float(r.max()), "median": float(r.median()), "fields": int(r.numel())}


def _per_field_rel_area(a, b, w):
    """relL2 per field of grids [field][lon][lat] with every point weighted by
    the Gauss weight of its latitude (the area-weighted variant)"""
    import torch

    sw = torch.as_tensor(w, dtype=a.dtype, device=a.device).sqrt()
    return _per_field_rel(a * sw, b * sw)


def run_ours(args, rank, world):
    import torch

    from sph_swe_b200 import build as b
    b.build()
    from sph_swe_b200 import capi

    dev = torch.device("cuda", rank % max(1, torch.cuda.device_count()))
    torch.cuda.set_device(dev)
    st = torch.cuda.current_stream()
    gl, gf, per_contr = cfg1_flops()
    flops_step = gl + gf
    spec, vort, div = _cfg1_inputs(dev, rank)
    forms = {"fp64": Cfg1(capi.SPH_PREC_FP64, dev, spec, vort, div),
             "mixed": Cfg1(capi.SPH_PREC_MIXED, dev, spec, vort, div)}
    for c in forms.values():
        for _ in range(args.warmup):
            c.step()
        c.sync_ok()
    torch.cuda.synchronize()

    # accuracy of the mixed form against the FP64 path (which matches the oracle
    # to 1e-12), per field: synthesis grids, analysis round trip, vector pair
    f64, mx = forms["fp64"], forms["mixed"]
    accuracy = {
        "scalar_synthesis_vs_fp64": _per_field_rel(mx.grid, f64.grid),
        "scalar_roundtrip_vs_input": _per_field_rel(mx.spec_out, spec),
        "vector_u_vs_fp64": _per_field_rel(mx.u, f64.u),
        "vector_v_vs_fp64": _per_field_rel(mx.v, f64.v),
        "vorticity_roundtrip_vs_input": _per_field_rel(mx.z, vort),
        "divergence_roundtrip_vs_input": _per_field_rel(mx.d, div),
        "fp64_scalar_roundtrip_vs_input": _per_field_rel(f64.spec_out, spec),
        "fp64_vorticity_roundtrip_vs_input": _per_field_rel(f64.z, vort),
        "scalar_synthesis_vs_fp64_area_weighted": _per_field_rel_area(mx.grid, f64.grid, mx.s.w),
        "vector_u_vs_fp64_area_weighted": _per_field_rel_area(mx.u, f64.u, mx.s.w),
        "vector_v_vs_fp64_area_weighted": _per_field_rel_area(mx.v, f64.v, mx.s.w),
    }
    # the forward vector transform alone: the mixed analysis of the FP64 grids
    # against the FP64 analysis of the same grids
    zm, dm = mx.s.vec_spat_to_SH(f64.u, f64.v)
    accuracy["vorticity_analysis_vs_fp64"] = _per_field_rel(zm, f64.z)
    accuracy["divergence_analysis_vs_fp64"] = _per_field_rel(dm, f64.d)
    del zm, dm

    ms = {}
    clocks = None
    for name in ("fp64", "mixed"):
        c = forms[name]
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        if name == "mixed":
            with ClockSampler(dev.index) as clk:
                ms[name] = _time(c.step, args.steps, st)
            clocks = clk.summary()
        else:
            ms[name] = _time(c.step, args.steps, st)
        c.sync_ok()
        if world > 1:
            torch.distributed.barrier()
        ms[name] = _max_over_ranks(ms[name], world, dev)
    value = flops_step * world / (ms["mixed"] * 1e-3) / 1e9
    value_fp64 = flops_step * world / (ms["fp64"] * 1e-3) / 1e9

    # Legendre stages timed alone on the same stream (64 scalar fields)
    leg = {}
    for name, c in forms.items():
        four = torch.empty(N_SCALAR, L_CFG1 + 1, c.s.nlat, dtype=torch.complex128, device=dev)
        for _ in range(3):
            c.s.legendre_synthesis(spec, four)
            c.s.legendre_analysis(four, c.spec_out)
        torch.cuda.synchronize()
        nrep = max(3, min(args.steps, 50))
        t_syn = _time(lambda: c.s.legendre_synthesis(spec, four), nrep, st) * 1e-3
        t_ana = _time(lambda: c.s.legendre_analysis(four, c.spec_out), nrep, st) * 1e-3
        c.sync_ok()
        leg[name] = {"synthesis_us": t_syn * 1e6, "analysis_us": t_ana * 1e6,
                     "synthesis_tflops": per_contr * N_SCALAR / t_syn / 1e12,
                     "analysis_tflops": per_contr * N_SCALAR / t_ana / 1e12}
        # the small batches of the RK4 stages (first fields of the same spectra;
        # mixed handle: variants autotuned per batch): synthesis / analysis us
        small = {}
        for nb in (1, 2, 4, 8):
            if name == "mixed":
                c.s.autotune(nb)
            sp, fo, so = spec[:nb], four[:nb], c.spec_out[:nb]
            c.s.legendre_synthesis(sp, fo)
            c.s.legendre_analysis(fo, so)
            t1 = _time(lambda: c.s.legendre_synthesis(sp, fo), nrep, st) * 1e3
            t2 = _time(lambda: c.s.legendre_analysis(fo, so), nrep, st) * 1e3
            small[str(nb)] = [_sig(t1), _sig(t2)]
        c.sync_ok()
        leg[name]["small_batches_us_syn_ana"] = small
        del four
    # the dominant stage, the int8 Legendre analysis (B preparation + contraction
    # of 64 fields): its tensor work is a few microseconds at int8 rate, so it is
    # bounded by HBM; achieved = its algorithmic bytes / its event-timed duration
    peaks, src = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = ana64_bytes() / (leg["mixed"]["analysis_us"] * 1e-6) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_i8b_prep_ana<32> + k_legendre_i8b<AnaI8<32>> (int8 Legendre analysis, "
                                          "64 fields, T255)",
                "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": args.traffic if args.traffic is not None else TRAFFIC_ANA64,
                "algorithmic_bytes": ana64_bytes(),
                "peak_source": f"HBM copy bandwidth of MEASURED_PEAKS.json ({src}); traffic = DRAM bytes of the two "
                               "launches from one ncu capture",
                "legendre": leg}

    # end-to-end through the C ABI with host buffers (mixed form): H2D of the
    # input spectra, the step, D2H of the output spectra
    h_spec = torch.from_numpy(random_spec(L_CFG1, N_SCALAR, 1 + rank)).pin_memory()
    h_vort = torch.from_numpy(random_spec(L_CFG1, N_PAIRS, 1001 + rank, zero_mean=True)).pin_memory()
    h_div = torch.from_numpy(random_spec(L_CFG1, N_PAIRS, 2001 + rank, zero_mean=True)).pin_memory()
    o_spec = torch.empty_like(h_spec).pin_memory()
    o_vort = torch.empty_like(h_vort).pin_memory()
    o_div = torch.empty_like(h_div).pin_memory()
    h2d = (h_spec.numel() + h_vort.numel() + h_div.numel()) * 16
    d2h = h2d

    def e2e_step():
        spec.copy_(h_spec, non_blocking=True)
        vort.copy_(h_vort, non_blocking=True)
        div.copy_(h_div, non_blocking=True)
        mx.step()
        o_spec.copy_(mx.spec_out, non_blocking=True)
        o_vort.copy_(mx.z, non_blocking=True)
        o_div.copy_(mx.d, non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    ms_e2e_serial = _max_over_ranks(_time(e2e_step, args.steps, st), world, dev)

    # the same steps pipelined: three streams (upload, compute, download) and two
    # device buffer sets, so that the upload of step k + 1 and the download of
    # step k - 1 overlap the compute of step k; every step still copies its own
    # inputs from pinned host memory and its results back
    ms_e2e = _max_over_ranks(_e2e_pipelined(mx.s, h_spec, h_vort, h_div, o_spec, o_vort, o_div, args.steps, dev),
                             world, dev)
    e2e_value = flops_step * world / (ms_e2e * 1e-3) / 1e9
    for c in forms.values():
        c.s.close()
    del forms, f64, mx, spec, vort, div
    torch.cuda.empty_cache()

    extra = {"fp64_form": {"value": value_fp64, "unit": "GFLOP/s", "ms_per_step": ms["fp64"]},
             "mixed_over_fp64": ms["fp64"] / ms["mixed"]}
    if not args.quick:
        extra["rk4"] = rk4_rates(dev, args)
        extra["rexi"] = rexi_rates(dev, args)
        extra["ensemble"] = ensemble_rates(dev, args)
        extra["T1023"] = t1023_rates(dev, args)
    return dict(value=value, ms=ms["mixed"], roofline=roofline, clocks=clocks,
                e2e={"value": e2e_value, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                     "ms_per_step": ms_e2e, "pipelined": "upload / compute / download streams, two buffer sets",
                     "ms_per_step_serial": ms_e2e_serial},
                launches=Cfg1.LAUNCHES * args.steps, accuracy=accuracy, extra=extra)


def _bump_state(s, dev, h0=1e4, amp=500.0):
    import torch

    lat0, lon0 = np.deg2rad(30.0), np.deg2rad(60.0)

    def bump(lon, mu):
        p = np.arcsin(mu)
        c = np.sin(p) * np.sin(lat0) + np.cos(p) * np.cos(lat0) * np.cos(lon - lon0)
        return h0 + amp * np.exp(-(np.arccos(np.clip(c, -1, 1)) / 0.1) ** 2)

    st = torch.zeros(3, s.nlm, dtype=torch.complex128, device=dev)
    st[0] = s.spat_to_SH(torch.from_numpy(s.grid_from(bump)).to(dev))
    return st


def rk4_rates(dev, args):
    """Nonlinear RK4 steps/s at T255 and at the T63 plain-method configuration,
    FP64 and mixed form, with the relative L2 of the mixed state against the
    FP64 state after the same steps."""
    import torch

    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    # T255: the reference's non-Robert advective form is unstable at dt = 30 s
    # (the oracle diverges within 60 steps); dt = 10 s with the reference's
    # default viscosity 1e5 runs stably.  T63: the plain-method configuration.
    # T255_vort_div: the vorticity-divergence form (state [h, zeta, delta]),
    # stable at dt = 60 s without viscosity.
    out = {}
    for key, L, dt, visc, n, form in (("T255", 255, 10.0, 1e5, 50, 1), ("T63", 63, 120.0, 0.0, 200, 1),
                                      ("T255_vort_div", 255, 60.0, 0.0, 50, 2)):
        res = {}
        states = {}
        s0 = Sph(L)
        st0 = _bump_state(s0, dev)  # one initial state (FP64 analysis) for both forms
        s0.close()
        for name, prec in (("fp64", capi.SPH_PREC_FP64), ("mixed", capi.SPH_PREC_MIXED)):
            s = Sph(L, precision=prec)
            for b in Sph.rk4_batches(1, form):  # kernel variants per batch (untimed set-up)
                s.autotune(b)
            p = Sph.swe_params(radius=6.371e6, dt=dt, viscosity=visc, nonlinear=form)
            st = st0.clone()
            s.swe_rk4(p, st, 3)
            torch.cuda.synchronize()
            st = st0.clone()
            ms = _time(lambda: s.swe_rk4(p, st, n), 1, torch.cuda.current_stream()) / n
            capi.check(capi.lib().sph_sync(s.h, None))
            states[name] = st
            launches = capi.lib().sph_swe_rk4_launches(s.h)
            res[name] = {"steps_per_s": 1000.0 / ms, "ms_per_step": ms, "kernel_launches_per_step": launches}
            s.close()
        names = ("h", "u", "v") if form == 1 else ("h", "vorticity", "divergence")
        rel = {q: float(torch.linalg.vector_norm(states["mixed"][k] - states["fp64"][k]) /
                        max(float(torch.linalg.vector_norm(states["fp64"][k])), 1e-300)) for k, q in enumerate(names)}
        out[key] = {**res, "mixed_over_fp64": res["mixed"]["steps_per_s"] / res["fp64"]["steps_per_s"],
                    "nsteps": n, "dt": dt, "viscosity": visc, "mixed_rel_l2_vs_fp64_after_nsteps": rel,
                    "kernel_launches_per_step": launches}
    return out


def rexi_rates(dev, args):
    """REXI configuration: T127 192x384, Robert linear SWE about h0 = 1e4 m,
    Gaussian-approximation REXI h = 0.2, M = 256 (535 poles), tau = 3600 s,
    24 steps from the Gaussian bump; FP64 direct and the mixed form (complex
    FP32 factors stored per plan, one FP64 refinement step), with the
    relative L2 of the mixed state against the FP64 state."""
    import torch

    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph, rexi_coefficients

    s = Sph(127)
    a, br, _ = rexi_coefficients(0.2, 256, False)
    st0 = _bump_state(s, dev)
    n = 24
    out, states = {}, {}
    for name, prec in (("fp64", capi.SPH_PREC_FP64), ("mixed", capi.SPH_PREC_MIXED)):
        rx = s.rexi(a, br, radius=6.371e6, tau=3600.0, precision=prec)
        st = st0.clone()
        rx.step(st, 2)  # warm-up; also the accuracy sample (see below)
        states[name] = st
        torch.cuda.synchronize()
        st = st0.clone()
        ms = _time(lambda: rx.step(st, n), 1, torch.cuda.current_stream()) / n
        capi.check(capi.lib().sph_sync(s.h, None))
        out[name] = {"steps_per_s": 1000.0 / ms, "ms_per_step": ms}
        rx.close()
    rel = {q: float(torch.linalg.vector_norm(states["mixed"][k] - states["fp64"][k]) /
                    max(float(torch.linalg.vector_norm(states["fp64"][k])), 1e-300)) for k, q in enumerate("huv")}
    s.close()
    # the reference's Robert REXI integration is not stable over many steps at
    # this size (the oracle grows without bound as well): accuracy after 2 steps
    return {"T127_M256": {**out, "poles": int(len(a)), "nsteps": n, "tau": 3600.0,
                          "mixed_over_fp64": out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"],
                          "mixed_rel_l2_vs_fp64_after_2_steps": rel}}


def t1023_rates(dev, args):
    """T1023 configuration: 1536 x 3072 Gauss grid, full nonlinear equations in
    vorticity-divergence form with Robert velocities on the grid, zonal jet
    80 sech^2((phi - 45 deg)/0.1) m/s with h in gradient-wind balance (mean
    1e4 m) plus a 120 m bump at (30N, 60E), dt = 15 s, 50 steps; FP64 and
    mixed form; relative L2 of h and vorticity of the mixed form against the
    FP64 form, and the mass drift (Y_00 of h) of each."""
    import torch

    from sph_swe_b200 import capi, scenarios
    from sph_swe_b200.sph import Sph

    L, n, dt, a = 1023, 50, 15.0, 6.371e6
    res, states = {}, {}
    st0 = None
    for name, prec in (("fp64", capi.SPH_PREC_FP64), ("mixed", capi.SPH_PREC_MIXED)):
        s = Sph(L, precision=prec)
        if st0 is None:
            h, u, v = scenarios.sech2_jet(s, radius=a, bump_amp=120.0)
            c = torch.from_numpy(np.cos(s.lat)).to(dev)[None, :]
            z, d = s.vec_spat_to_SH(torch.from_numpy(u[None]).to(dev) * c, torch.from_numpy(v[None]).to(dev) * c,
                                    robert=True)
            st0 = torch.stack([s.spat_to_SH(torch.from_numpy(h).to(dev)), z[0] / a, d[0] / a])
        p = Sph.swe_params(radius=a, dt=dt, nonlinear=2)
        for b in Sph.rk4_batches(1, 2):  # kernel variants per batch (untimed set-up)
            s.autotune(b)
        st = st0.clone()
        s.swe_rk4(p, st, 3)
        torch.cuda.synchronize()
        st = st0.clone()
        ms = _time(lambda: s.swe_rk4(p, st, n), 1, torch.cuda.current_stream()) / n
        capi.check(capi.lib().sph_sync(s.h, None))
        m0, m1 = st0[0, 0].real.item(), st[0, 0].real.item()
        res[name] = {"steps_per_s": 1000.0 / ms, "ms_per_step": ms, "mass_drift_rel": abs(m1 - m0) / abs(m0)}
        launches = capi.lib().sph_swe_rk4_launches(s.h)
        states[name] = st
        s.close()
    rel = {q: float(torch.linalg.vector_norm(states["mixed"][k] - states["fp64"][k]) /
                    torch.linalg.vector_norm(states["fp64"][k])) for k, q in enumerate(("h", "vorticity", "divergence"))}
    out = {**res, "mixed_over_fp64": res["mixed"]["steps_per_s"] / res["fp64"]["steps_per_s"], "nsteps": n, "dt": dt,
           "grid": "1536 x 3072", "form": "nonlinear, vorticity-divergence with Robert velocities",
           "mixed_rel_l2_vs_fp64_after_nsteps": rel, "kernel_launches_per_step": launches}
    del states, st0
    torch.cuda.empty_cache()
    return out


ENSEMBLE = ((31, 96), (63, 96), (127, 48), (255, 16))
ENSEMBLE_STEPS = 100


def _random_bumps(s, n, rng, h0=1e4):
    """n grids h0 + A exp(-(d/sigma)^2): A ~ U(100, 800) m, centre uniform on
    the sphere (sin(lat) ~ U(-1, 1), lon ~ U(0, 2 pi)), sigma ~ U(0.05, 0.2) rad."""
    out = []
    for _ in range(n):
        amp, z, lon0, sig = rng.uniform(100, 800), rng.uniform(-1, 1), rng.uniform(0, 2 * np.pi), rng.uniform(0.05, 0.2)
        lat0 = np.arcsin(z)

        def f(lon, mu, lat0=lat0, lon0=lon0, amp=amp, sig=sig):
            p = np.arcsin(mu)
            c = np.sin(p) * np.sin(lat0) + np.cos(p) * np.cos(lat0) * np.cos(lon - lon0)
            return h0 + amp * np.exp(-(np.arccos(np.clip(c, -1, 1)) / sig) ** 2)

        out.append(s.grid_from(f))
    return np.stack(out)


def ensemble_rates(dev, args):
    """Ensemble configuration: 256 members (96 x T31, 96 x T63, 48 x T127,
    16 x T255), nonlinear RK4 with dt = 120 * 63 / T s, 100 steps, one CUDA
    graph replay per step for all members (each truncation on its own graph
    branch).  The members integrate the vorticity-divergence form: the
    reference's advective u, v form is unstable at T255 with dt = 29.6 s and no
    viscosity (the T255 group blows up within the 100 steps).  FP64 and mixed form; the FP64 form is also timed group by group
    (one batched graph per truncation, run one after another) to show what the
    branches overlap; the mixed state is compared with the FP64 state."""
    import torch

    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Ensemble, Sph

    rng = np.random.default_rng(20261203)
    init = {}
    for L, n in ENSEMBLE:
        s = Sph(L)
        st = torch.zeros(n, 3, s.nlm, dtype=torch.complex128, device=dev)
        st[:, 0] = s.spat_to_SH(torch.from_numpy(_random_bumps(s, n, rng)).to(dev))
        init[L] = st
        s.close()
    stream = torch.cuda.current_stream()
    out, finals = {}, {}
    for name, prec in (("fp64", capi.SPH_PREC_FP64), ("mixed", capi.SPH_PREC_MIXED)):
        groups = []
        for L, n in ENSEMBLE:
            s = Sph(L, precision=prec)
            for b in Sph.rk4_batches(n, 2):  # variants per truncation and batch (untimed set-up)
                s.autotune(b)
            groups.append((s, Sph.swe_params(radius=6.371e6, dt=120.0 * 63 / L, nonlinear=2), init[L].clone(), None))
        e = Ensemble(groups)
        e.step(3)
        for (_, _, st, _), (L, _) in zip(groups, ENSEMBLE):
            st.copy_(init[L])
        torch.cuda.synchronize()
        ms = _time(lambda: e.step(ENSEMBLE_STEPS), 1, stream) / ENSEMBLE_STEPS
        members = sum(n for _, n in ENSEMBLE)
        out[name] = {"member_steps_per_s": members * 1000.0 / ms, "ms_per_ensemble_step": ms,
                     "kernel_launches_per_step": e.launches}
        finals[name] = [g[2].clone() for g in groups]
        if name == "fp64":
            seq = 0.0
            for s, p, st, _ in groups:
                st.copy_(init[s.L])
                s.swe_rk4_batched(p, st, 3)  # one batched graph per truncation
                torch.cuda.synchronize()
                seq += _time(lambda: s.swe_rk4_batched(p, st, ENSEMBLE_STEPS), 1, stream) / ENSEMBLE_STEPS
            out[name]["ms_per_step_groups_one_after_another"] = seq
        e.close()
        for s, *_ in groups:
            s.close()
        del groups
    rel = {}
    for (L, n), a, b in zip(ENSEMBLE, finals["mixed"], finals["fp64"]):
        r = (torch.linalg.vector_norm(a - b, dim=2) / torch.linalg.vector_norm(b, dim=2)).max(dim=0).values
        rel[f"T{L}"] = {q: float(r[k]) for k, q in enumerate(("h", "vorticity", "divergence"))}
    out["members"] = {f"T{L}": n for L, n in ENSEMBLE}
    out["nsteps"] = ENSEMBLE_STEPS
    out["mixed_over_fp64"] = out["mixed"]["member_steps_per_s"] / out["fp64"]["member_steps_per_s"]
    out["mixed_max_rel_l2_vs_fp64_after_nsteps"] = rel
    del finals, init
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------ CPU baseline (oracle port)
class OracleCfg1:
    """The transform-throughput step on the host cores through the oracle
    (C++/OpenMP FP64 restatement of the reference's transforms; its vector
    pair through the oracle's restatement of the exact vector transforms):
    synthesis + analysis of the 64 scalar fields, vector synthesis of the 32
    vorticity/divergence pairs to (u, v) and vector analysis back, i.e. the
    same work and the same algorithmic flop count as one GPU step."""

    def __init__(self):
        from oracle import oracle as O
        from oracle.vortdiv import VortDiv

        O.build()
        self.O = O
        self.g = O.Grid(L_CFG1)
        self.vd = VortDiv(self.g)
        self.cos = np.sqrt(self.vd.c2)[None, :]
        self.spec = random_spec(L_CFG1, N_SCALAR, 1)
        self.vort = random_spec(L_CFG1, N_PAIRS, 1001, zero_mean=True)
        self.div = random_spec(L_CFG1, N_PAIRS, 2001, zero_mean=True)

    def step(self):
        g, vd = self.g, self.vd
        g.spat_to_SH(g.SH_to_spat(self.spec))
        for k in range(N_PAIRS):
            U, V = vd.vec_synthesis(self.vort[k], self.div[k])
            u, v = U / self.cos, V / self.cos
            vd.vec_analysis(u * self.cos, v * self.cos)

    def cores(self):
        return self.O.num_threads()


def cpu_baseline(min_seconds=12.0, max_steps=40):
    """Oracle restatement of the same step on the host cores, repeated until
    >= min_seconds (a bounded sample of the headline workload)."""
    c = OracleCfg1()
    c.step()
    steps = 0
    t0 = time.perf_counter()
    while steps < max_steps:
        c.step()
        steps += 1
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    flops = steps * sum(cfg1_flops()[:2])
    return {"value": flops / dt / 1e9, "unit": "GFLOP/s", "cores": c.cores(), "kind": "port",
            "sample": f"{steps} steps of the same workload (64 scalar fields + 32 vort/div pairs, inverse + forward, "
                      f"T255) through the oracle (C++/OpenMP FP64), {dt:.1f} s"}


def profile_case(which="all"):
    """One small instance of each workload, for ncu captures of every kernel
    family (no timing): transforms of 64 scalar fields at T255 in both forms,
    one nonlinear RK4 step at T255 (advective and vorticity-divergence forms),
    one REXI step at T127 (M = 64) and one spectral operator pass.  which:
    "all", or one workload alone: "cfg1" (two steps of the transform
    configuration in each form, built-in kernel variants), "specops" (the
    spectral operators on 256 T255 spectra), "rk4" (two
    nonlinear RK4 steps at T255 in each form, tuned variants), "fp64x64" (two
    inverse + forward transforms of the 64 scalar T255 fields in the FP64
    form), "mixed64" (two inverse + forward transforms
    of the 64 scalar T255 fields in the mixed form), "rexi" (two REXI steps at
    T127, M = 64, FP64 with stored factors, Robert form), "rexi_s0" (the same
    in the non-Robert form)."""
    import torch

    from sph_swe_b200 import build as b
    b.build()
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph, rexi_coefficients

    dev = torch.device("cuda", 0)
    if which == "cfg1":
        # two steps of the transform-throughput configuration in each form, with
        # the built-in kernel variants (the launch-list case)
        spec, vort, div = _cfg1_inputs(dev, 0)
        for prec in (capi.SPH_PREC_FP64, capi.SPH_PREC_MIXED):
            s = Sph(L_CFG1, precision=prec)
            grid = torch.empty(N_SCALAR, s.nphi, s.nlat, dtype=torch.float64, device=dev)
            for _ in range(2):
                s.spat_to_SH(s.SH_to_spat(spec, out=grid))
                s.vec_spat_to_SH(*s.vec_SH_to_spat(vort, div))
            capi.check(capi.lib().sph_sync(s.h, None))
            s.close()
        print(json.dumps({"profile_case": which}))
        return
    if which == "specops":
        # the spectral operators on 256 T255 spectra (135 MB, more than L2),
        # one launch each
        s = Sph(L_CFG1)
        spec = torch.from_numpy(random_spec(L_CFG1, 4 * N_SCALAR, 1)).to(dev)
        out = torch.empty_like(spec)
        for op in ("diff_lon", "d1mu2", "mu", "mu2", "laplace", "helmholtz"):
            s.spec_op(op, spec, a=1.0, b=2.0, out=out)
        capi.check(capi.lib().sph_sync(s.h, None))
        s.close()
        print(json.dumps({"profile_case": which}))
        return
    if which == "rk4":
        # two nonlinear RK4 steps at T255 (reference advective form, dt 10 s,
        # viscosity 1e5) in each form, kernel variants tuned per batch
        s0 = Sph(255)
        st0 = _bump_state(s0, dev)
        s0.close()
        for prec in (capi.SPH_PREC_FP64, capi.SPH_PREC_MIXED):
            s = Sph(255, precision=prec)
            for nb in Sph.rk4_batches(1, 1):
                s.autotune(nb)
            p = Sph.swe_params(radius=6.371e6, dt=10.0, viscosity=1e5, nonlinear=1)
            st = st0.clone()
            s.swe_rk4(p, st, 2)
            capi.check(capi.lib().sph_sync(s.h, None))
            s.close()
        print(json.dumps({"profile_case": which}))
        return
    if which in ("mixed64", "fp64x64"):
        s = Sph(L_CFG1, precision=capi.SPH_PREC_MIXED if which == "mixed64" else capi.SPH_PREC_FP64)
        spec = torch.from_numpy(random_spec(L_CFG1, N_SCALAR, 1)).to(dev)
        for _ in range(2):
            s.spat_to_SH(s.SH_to_spat(spec))
        capi.check(capi.lib().sph_sync(s.h, None))
        s.close()
        print(json.dumps({"profile_case": which}))
        return
    if which in ("rexi", "rexi_s0"):
        s = Sph(127)
        a, br, _ = rexi_coefficients(0.2, 64, False)
        rx = s.rexi(a, br, radius=6.371e6, tau=3600.0, robert=1 if which == "rexi" else 0)
        rx.step(_bump_state(s, dev), 2)
        torch.cuda.synchronize()
        rx.close()
        s.close()
        print(json.dumps({"profile_case": which}))
        return
    for prec in (capi.SPH_PREC_FP64, capi.SPH_PREC_MIXED):
        s = Sph(L_CFG1, precision=prec)
        spec = torch.from_numpy(random_spec(L_CFG1, N_SCALAR, 1)).to(dev)
        s.spat_to_SH(s.SH_to_spat(spec))
        st = _bump_state(s, dev)
        for form in (1, 2):
            s.swe_rk4(Sph.swe_params(radius=6.371e6, dt=10.0, viscosity=1e5, nonlinear=form), st.clone(), 1)
        capi.check(capi.lib().sph_sync(s.h, None))
        s.close()
    s = Sph(L_CFG1)
    x = torch.from_numpy(random_spec(L_CFG1, N_SCALAR, 2)).to(dev)
    s.spec_op("laplace", x)
    s.close()
    s = Sph(127)
    a, br, _ = rexi_coefficients(0.2, 64, False)
    rx = s.rexi(a, br, radius=6.371e6, tau=3600.0)
    rx.step(_bump_state(s, dev), 1)
    torch.cuda.synchronize()
    rx.close()
    s.close()
    print(json.dumps({"profile_case": "done"}))


def run_reference(args, rank, world):
    """CPU arm: the oracle (C++/OpenMP FP64 restatement; the reference's own
    SHTNS/FFTW/LAPACK build is unavailable on this machine) on all host cores,
    on the same step as our arm: 64 scalar T255 fields and 32 vort/div pairs,
    inverse + forward (the vector pair through the oracle's exact vector
    transforms)."""
    if rank != 0:
        return None
    c = OracleCfg1()
    for _ in range(args.warmup):
        c.step()
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        c.step()
        ts.append(time.perf_counter() - t0)
    dt = float(np.mean(ts))
    value = sum(cfg1_flops()[:2]) / dt / 1e9
    sample = ("per step inverse + forward of the 64 scalar T255 fields and the 32 vort/div pairs (oracle C++/OpenMP "
              "FP64; the reference's SHTNS/FFTW/LAPACK build is unavailable on this machine)")
    return {"metric": METRIC, "value": value, "unit": "GFLOP/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "SHT throughput: T255 384x768 Gauss grid, 64 scalar fields + 32 vort/div pairs, "
                                   "inverse + forward per step", "lmax": L_CFG1, "nlat": 384, "nphi": 768,
                       "fields": N_SCALAR, "vector_pairs": N_PAIRS, "gflop_per_step": sum(cfg1_flops()[:2]) / 1e9},
            "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": c.cores(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _sig(x, n=3):
    return float(f"{x:.{n}g}") if isinstance(x, (int, float)) and x == x else x


def summary(line):
    """The figures a reader needs, in a compact object printed LAST in the
    line (the driver keeps the tail of the output): the FP64 form of the
    headline step, every mixed/FP64 speed ratio, the worst per-field relative
    L2 of the mixed form, and the Legendre kernel times."""
    out = {"fp64_form_gflops": _sig(line.get("fp64_form", {}).get("value", float("nan")), 5),
           "fp64_form_ms": _sig(line.get("fp64_form", {}).get("ms_per_step", float("nan")), 4),
           "mixed_ms": _sig(line["ms_per_step"], 4)}
    ratios = {"cfg1": line.get("mixed_over_fp64")}
    for k, v in line.get("rk4", {}).items():
        ratios["rk4_" + k] = v.get("mixed_over_fp64")
    for k, v in line.get("rexi", {}).items():
        ratios["rexi_" + k] = v.get("mixed_over_fp64")
    if "ensemble" in line:
        ratios["ensemble"] = line["ensemble"].get("mixed_over_fp64")
    if "T1023" in line:
        ratios["T1023"] = line["T1023"].get("mixed_over_fp64")
    out["mixed_over_fp64"] = {k: _sig(v) for k, v in ratios.items() if v is not None}
    acc = line.get("accuracy", {})
    out["mixed_cfg1_max_rel_l2"] = {k.replace("_vs_fp64", "").replace("_vs_input", ""): _sig(v["max"], 2)
                                    for k, v in acc.items() if not k.startswith("fp64") and "area" not in k}
    runs = {}
    for k, v in line.get("rk4", {}).items():
        runs["rk4_" + k] = v.get("mixed_rel_l2_vs_fp64_after_nsteps")
    if "T1023" in line:
        runs["T1023"] = line["T1023"].get("mixed_rel_l2_vs_fp64_after_nsteps")
    out["mixed_run_rel_l2"] = {k: {q: _sig(x, 2) for q, x in v.items()} for k, v in runs.items() if v}
    leg = line.get("roofline", {}).get("legendre", {})
    out["legendre_us_syn_ana"] = {k: [_sig(v["synthesis_us"]), _sig(v["analysis_us"])] for k, v in leg.items()}
    out["roofline_frac"] = _sig(line.get("roofline", {}).get("frac", float("nan")))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quick", action="store_true", help="skip the RK4 side measurements")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu DRAM bytes per launch of the dominant kernel (default: the committed capture)")
    ap.add_argument("--profile-case", nargs="?", const="all", default=None,
                    help="run one small instance of each workload (for ncu); optionally one of cfg1, specops, rk4, fp64x64, mixed64, rexi, rexi_s0")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res))
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
        return

    r = run_ours(args, rank, world)
    if rank == 0:
        line = {
            "metric": METRIC, "value": r["value"], "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (Legendre GEMMs int8 integer split, exact int32 sums, one f64 combination per tile)",
            "data": "synthetic",
            "config": {"workload": "SHT throughput: T255 384x768 Gauss grid, 64 scalar fields + 32 vort/div pairs, "
                                   "inverse + forward per step, mixed-precision form",
                       "lmax": L_CFG1, "nlat": 384, "nphi": 768, "fields": N_SCALAR, "vector_pairs": N_PAIRS,
                       "gflop_per_step": sum(cfg1_flops()[:2]) / 1e9,
                       "l2": "inputs larger than L2 (>= 270 MB touched per step); no flush"},
            "roofline": r["roofline"], "clocks": r["clocks"], "e2e": r["e2e"], "gpu_launches": r["launches"],
            "accuracy": r["accuracy"],
        }
        if not args.quick:
            line["cpu_baseline"] = cpu_baseline()
        line.update(r["extra"])
        line["summary"] = summary(line)
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
