"""Benchmark of the B200 H*psi sweep (RSPACE kukan hot path).

Workload (Si512): 4x4x4 diamond supercell of silicon, a = 41.04 bohr, 128^3
grid (h = 0.3206 bohr), 512 atoms jittered by sigma = 0.05 bohr (seed 4),
1100 bands, Si PAW projector tables (12 projectors per atom), FP32 psi.  One
step applies the fused H (stencil + veff + nonlocal D term, with stored
<p|psi>) to all 1100 bands -- kukan's rayleighritz_hamiltonian sweep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  --impl reference times the CPU oracle (the
FP64 restatement of kukan's loops) on this host's cores on a bounded sample
of the same sweep.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NB = 1100
GRID = 128
A_SI = 10.26
NCELL = 4
SIGMA, SEED = 0.05, 4
E2E_BANDS = 128
CPU_SAMPLE_BANDS = None  # one band per host thread (4..64)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_cell(list_builder=None):
    from rspacedist_b200 import system as S
    ds = S.load_dataset("si_paw")
    pos = S.diamond_positions(NCELL, A_SI, SIGMA, SEED)
    return S.make_cell(NCELL * A_SI, GRID, pos, ds, list_builder=list_builder)


def oracle_lists(atoms, rcut, nmax, h, npmax, nfdg, num_list):
    """The list vectors of pseudocalc_01b from the CPU oracle (the reference
    arm builds its cell with these, so it never loads the CUDA library)."""
    from oracle import oracle as O
    st, d = O.sphere_lists(atoms, rcut, nmax, h, npmax, nfdg, num_list)
    if st != 0:
        raise RuntimeError(f"oracle sphere_lists status {st}")
    return (d["natx"], d["naty"], d["natz"], d["natinf"], d["lst"], d["lstx"], d["lsty"],
            d["lstz"])


# DRAM bytes (read + write) of one stencil launch on the Si512 grid per band:
# ncu dram__bytes_read.sum + dram__bytes_write.sum of a 200-band launch, from
# the profile summary named beside it (capture command and per-launch figures
# there); None where no capture exists.
STENCIL_TRAFFIC_PER_BAND = {
    "k_stencil_f32_zmarch": ((1905046016 + 1640433920) / 200,
                             "profiles/stencil_f32_zmarch_si512.md"),
    "k_stencil_f32_tma": ((1842567936 + 1636464384) / 200,
                          "profiles/stencil_f32_tma_si512.md"),
}


def algorithmic_bytes(cell, nb, entries, s=4, s_p=4):
    """Bytes a perfect H*psi sweep must move: psi read + hpsi write, veff,
    the nonzero projector entries (values + atom index) and the inverse-list
    offsets, each once per call."""
    N = cell.N
    return N * nb * 2 * s + N * s + entries * (cell.nprjmx * s_p + 4) + (N + 1) * 4


def measured_peak():
    for p in (os.path.join(ROOT, "MEASURED_PEAKS.json"),):
        if os.path.exists(p):
            d = json.load(open(p))
            return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock, its maximum, power and the clock-event reasons of this
    process's GPU, read through NVML every 5 ms while the timed region runs
    (nvidia-smi every 200 ms when NVML is not importable).  Reads only."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index=0):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, set of reasons)
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.index).uuid)
        h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        return pynvml, h

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _poll_nvml(self):
        nv, h = self.nvml
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self.stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = get_reasons(h)
                self.samples.append((sm, mx, {n for n, b in zip(self.NAMES, bits) if r & b}))
            except Exception:
                pass
            self.stop.wait(0.005)

    def _read_smi(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) >= 9 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                self.samples.append((float(r[1]), float(r[2]),
                                     {n for n, v in zip(self.NAMES, r[5:9])
                                      if v.lower() == "active"}))

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.nvml or self.proc:
            self.t.join(timeout=5)

    def summary(self):
        sm = [x[0] for x in self.samples]
        reasons = set()
        for x in self.samples:
            reasons |= x[2]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(x[1] for x in self.samples) if sm else None,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "source": "nvml" if self.nvml else "nvidia-smi"}


def set_staging(g, staging, nb):
    """Selects the FP32 stencil's plane staging on geometry g ("tma" or "cp");
    True when nb-band calls run the TMA form."""
    import ctypes as C
    from rspacedist_b200 import lib as RL
    tma = C.c_int(0)
    mode = {"tma": 0, "cp": 1}[staging]
    RL.call("rs_hpsi_f32_staging", g.handle, mode, nb, C.byref(tma))
    return bool(tma.value)


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from rspacedist_b200 import kukan as K

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)

    t0 = time.time()
    cell = make_cell()
    g = K.Geometry(cell)
    tma = set_staging(g, args.staging, args.bands)
    stencil_kernel = "k_stencil_f32_tma" if tma else "k_stencil_f32_zmarch"
    log(f"[rank {rank}] set-up {time.time() - t0:.1f}s  entries={g.entries} "
        f"num_list={cell.num_list} natinf={int(cell.natinf.mean())}")
    from rspacedist_b200 import system as S
    veff = torch.tensor(S.smooth_veff(cell, 1), dtype=torch.float32, device=dev)
    dij = torch.tensor(cell.dij, dtype=torch.float64, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    nb = args.bands
    psi = torch.randn((nb, cell.N), generator=gen, dtype=torch.float32, device=dev) * 0.1
    rp = K.nonlocaloperation_01(g, psi)
    hpsi = torch.empty_like(psi)
    nbytes = algorithmic_bytes(cell, nb, g.entries)
    stream = torch.cuda.current_stream()

    def step():
        K.hpsi(g, veff, dij, rp, psi, out=hpsi)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    import ctypes as C
    from rspacedist_b200 import lib as RL
    chunk, nlb = C.c_int(0), C.c_int(0)
    RL.call("rs_hpsi_f32_tuning", g.handle, C.byref(chunk), C.byref(nlb))
    nl_chunk = chunk.value
    nchunks = 1 if nl_chunk <= 0 else -(-nb // nl_chunk)
    launches_per_step = 1 + 2 * nchunks  # k_tcoef_f32, then stencil + nonlocal per chunk
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if args.profile_range == "sweep":
            torch.cuda.cudart().cudaProfilerStart()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        if args.profile_range == "sweep":
            torch.cuda.cudart().cudaProfilerStop()
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
        dist.barrier()
    value = nbytes * world / (ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    sweep_gbs = nbytes / (ms * 1e-3) / 1e9

    # The dominant kernel of the sweep (about half of its time) is the stencil
    # k_stencil_f32_zmarch.  It is timed on its own over the same steps: the
    # same call on the same bands with a geometry that has no atoms, so
    # rs_hpsi_f32 launches the stencil and nothing else.
    import types
    g0 = K.Geometry(types.SimpleNamespace(
        shape=cell.shape, h=cell.h, natom=0, nprjmx=cell.nprjmx, num_list=1, N=cell.N,
        nprj=np.zeros(1, np.int32), natinf=np.zeros(1, np.int32), lst=np.zeros(1, np.int32),
        vnlocp=np.zeros(1)))
    set_staging(g0, args.staging, nb)
    rp0 = torch.zeros(1, dtype=torch.float64, device=dev)
    for _ in range(args.warmup):
        K.hpsi(g0, veff, dij, rp0, psi, out=hpsi)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    es0, es1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.profile_range == "stencil":
        torch.cuda.cudart().cudaProfilerStart()
    es0.record(stream)
    for _ in range(args.steps):
        K.hpsi(g0, veff, dij, rp0, psi, out=hpsi)
    es1.record(stream)
    torch.cuda.synchronize()
    if args.profile_range == "stencil":
        torch.cuda.cudart().cudaProfilerStop()
    st_ms = es0.elapsed_time(es1) / args.steps
    if world > 1:
        t = torch.tensor([st_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        st_ms = t.item()
    st_bytes = cell.N * nb * 8 + cell.N * 4  # psi read, hpsi write, veff
    st_gbs = st_bytes / (st_ms * 1e-3) / 1e9
    g0.close()

    # the plain FP64 drop-in path on the same sweep (rs_hpsi_f64: FP64 psi,
    # veff and tables), for an FP64-to-FP64 comparison with the CPU oracle
    fp64 = None
    if args.fp64_sweep:
        psi64 = psi.double()
        veff64 = veff.double()
        rp64 = K.nonlocaloperation_01(g, psi64)
        h64 = torch.empty_like(psi64)
        for _ in range(args.warmup):
            K.hpsi(g, veff64, dij, rp64, psi64, out=h64)
        torch.cuda.synchronize()
        ef0, ef1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ef0.record(stream)
        for _ in range(args.steps):
            K.hpsi(g, veff64, dij, rp64, psi64, out=h64)
        ef1.record(stream)
        torch.cuda.synchronize()
        f_ms = ef0.elapsed_time(ef1) / args.steps
        b64 = algorithmic_bytes(cell, nb, g.entries, s=8, s_p=8)
        fp64 = {"ms_per_step": round(f_ms, 3), "gbs": round(b64 / (f_ms * 1e-3) / 1e9, 1),
                "band_points_per_s": round(nb * cell.N / (f_ms * 1e-3), 1),
                "algorithmic_bytes_per_step": b64, "entry_point": "rs_hpsi_f64"}
        del psi64, veff64, rp64, h64
        torch.cuda.empty_cache()

    step()  # hpsi holds the sweep's output again (the stencil-only run wrote it)
    # end to end through the host-buffer entry point: every band of the sweep
    # from pinned host memory and back (rs_hpsi_host_f32), when the host has
    # room for the two pinned copies
    ne = nb if host_bytes_available() > 3 * 2 * nb * cell.N * 4 else min(E2E_BANDS, nb)
    hin = torch.empty((ne, cell.N), dtype=torch.float32, pin_memory=True)
    hin.copy_(psi[:ne])
    hout = torch.empty_like(hin, pin_memory=True)
    rp_e = rp[:ne].contiguous()
    for _ in range(2):
        K.hpsi_host(g, veff, dij, rp_e, hin, hout, chunk=32)
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(e2e_steps):
        K.hpsi_host(g, veff, dij, rp_e, hin, hout, chunk=32)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - e0) / e2e_steps
    e2e_bytes = algorithmic_bytes(cell, ne, g.entries)
    e2e_gbs = e2e_bytes / e2e_s / 1e9
    h2d_bytes, d2h_bytes = int(hin.numel() * 4), int(hout.numel() * 4)
    e2e_ok = bool(torch.equal(hout[:8].to(dev), hpsi[:8]))
    del hin, hout, rp_e

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sample = cpu_sample(cell)
        cpu = cpu_baseline(cell, sample)
        parity = check_parity(cell, g, dij, sample)
    scf_out = scf64_out = None
    if rank == 0 and world == 1 and args.scf_loops > 0:
        del psi, hpsi, rp
        torch.cuda.empty_cache()
        scf_out = run_scf_leg(cell, args.scf_loops)
        scf64_out = run_scf_si64(args.scf_loops)
    traffic_pb, traffic_src = STENCIL_TRAFFIC_PER_BAND[stencil_kernel]
    if rank == 0:
        out = {
            "metric": "Si512 H*psi sweep HBM GB/s (FP32 psi); SCF time to eps in 'scf'",
            "value": round(value, 1), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Si512 geometry, random psi, synthetic smooth veff)",
            "config": {"workload": "Si512 H*psi sweep: 128^3 grid, 1100 bands, 512 Si atoms "
                                   "x 12 projectors, FP32 psi, stored <p|psi>",
                       "grid": [GRID] * 3, "bands": nb, "atoms": cell.natom,
                       "projectors": cell.nprjmx, "inverse_entries": g.entries,
                       "l2": "inputs (9.2 GB psi) larger than L2; no flush",
                       "nl_band_chunk": nl_chunk, "nl_bands_per_thread": nlb.value,
                       "stencil_staging": "tma" if tma else "cp.async",
                       "parallelism": f"bands replicated per GPU x{world}"},
            "band_points_per_s": round(nb * cell.N * world / (ms * 1e-3), 1),
            "roofline": {"bound": "hbm", "kernel": stencil_kernel,
                         "achieved": round(st_gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(st_gbs / peak, 4),
                         "traffic": (round(traffic_pb * nb) if traffic_pb else None),
                         "traffic_source": (f"{traffic_src}: ncu dram__bytes_read.sum + "
                                            "dram__bytes_write.sum of one 200-band launch, "
                                            "scaled by bands" if traffic_pb else None),
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": st_bytes,
                         "ms_per_launch": round(st_ms, 3)},
            "roofline_sweep": {"bound": "hbm",
                               "kernels": f"k_tcoef_f32, then {stencil_kernel} and "
                                          "k_nl_rmw_f32 per band chunk",
                               "achieved": round(sweep_gbs, 1), "peak": peak, "unit": "GB/s",
                               "frac": round(sweep_gbs / peak, 4),
                               "algorithmic_bytes_per_step": nbytes},
            "e2e": {"value": round(e2e_gbs, 2), "unit": "GB/s",
                    "h2d_bytes_per_step": h2d_bytes,
                    "d2h_bytes_per_step": d2h_bytes,
                    "bands": ne, "entry_point": "rs_hpsi_host_f32",
                    "equals_device_sweep": e2e_ok},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(),
        }
        if cpu:
            out["cpu_baseline"] = cpu
        if parity:
            out["parity"] = parity
        if fp64:
            out["fp64_sweep"] = fp64
        if scf_out:
            out["scf"] = scf_out
        if scf64_out:
            out["scf_si64"] = scf64_out
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


SCF_EPS_CHARGE = 1e-6      # kukan's diff_charge stopping rule
SCF_EPS_ENERGY = 2e-8      # Ha/atom change of the free energy over one iteration
SCF_ETA, SCF_NBRYDN = 0.3, 40


def run_scf_pair(cell, M, nocc, looplimit, ncgscf):
    """kukan's SCF of `cell` on the mixed path (FP32 bands, FP64 polish) and
    on the plain FP64 path from the same seeded smooth random bands, each
    until diff_charge < SCF_EPS_CHARGE and the free energy changed by less
    than SCF_EPS_ENERGY per atom over the last iteration.  The loop's wall
    time is taken with the device synchronised; the set-up (local potential,
    start bands, their orthonormalisation, the start density) is reported
    apart."""
    import torch
    from rspacedist_b200 import lib, scf
    prm = lib.solver_prm(ncgscf=ncgscf)
    res = {}
    for name, dt in (("mixed", torch.float32), ("fp64", torch.float64)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = scf.run_scf(cell, M, nocc, dtype=dt, prm=prm, looplimit=looplimit, eta=SCF_ETA,
                        nbrydn=SCF_NBRYDN, eps_scf=SCF_EPS_CHARGE, eps_energy=SCF_EPS_ENERGY,
                        profile=True, start="random", seed=0)
        total = time.perf_counter() - t0
        r.bands = r.rho_out = None
        res[name] = (r, total)
        torch.cuda.empty_cache()
        log(f"[scf] {cell.natom} atoms {name}: converged {r.converged} in {r.iterations} "
            f"iterations, {r.seconds:.2f} s (+{total - r.seconds:.2f} s set-up); "
            f"F {r.energy['free']:.8f}")
    (a, ta), (b, tb) = res["mixed"], res["fp64"]
    per_it = lambda r: r.seconds / max(1, r.iterations)
    tail = lambda r: (abs(r.energies[-1] - r.energies[-2]) / cell.natom
                      if len(r.energies) > 1 else None)
    return {
        "eps": {"diff_charge": SCF_EPS_CHARGE,
                "free_energy_change_ha_per_atom_per_iteration": SCF_EPS_ENERGY},
        "converged": {"mixed": a.converged, "fp64": b.converged},
        "iterations": {"mixed": a.iterations, "fp64": b.iterations},
        "time_to_eps_s": {"mixed": round(a.seconds, 2), "fp64": round(b.seconds, 2)},
        "setup_s": {"mixed": round(ta - a.seconds, 2), "fp64": round(tb - b.seconds, 2)},
        "speedup_time_to_eps_mixed_vs_fp64": round(b.seconds / a.seconds, 3),
        "s_per_iter": {"mixed": round(per_it(a), 3), "fp64": round(per_it(b), 3)},
        "free_energy_ha": {"mixed": a.energy["free"], "fp64": b.energy["free"]},
        "etot_ha": {"mixed": a.energy["total"], "fp64": b.energy["total"]},
        "etot_diff_ha_per_atom": abs(a.energy["total"] - b.energy["total"]) / cell.natom,
        "free_energy_diff_ha_per_atom": abs(a.energy["free"] - b.energy["free"]) / cell.natom,
        "last_step_change_ha_per_atom": {"mixed": tail(a), "fp64": tail(b)},
        "energy_terms_fp64": b.energy,
        "max_abs_occupied_eig_diff_ha": float(np.abs(np.sort(a.sval)[:nocc]
                                                     - np.sort(b.sval)[:nocc]).max()),
        "mixed_phase_s": {k: round(v, 3) for k, v in a.phase_seconds.items()},
        "fp64_phase_s": {k: round(v, 3) for k, v in b.phase_seconds.items()},
        "diff_charge_mixed": [float(f"{d:.3e}") for d in a.diff],
        "diff_charge_fp64": [float(f"{d:.3e}") for d in b.diff],
        "free_energy_mixed": [round(e, 8) for e in a.energies],
        "free_energy_fp64": [round(e, 8) for e in b.energies],
        "timing": "wall clock of the SCF loop (iteration 1 to the stopping rule, the mixed "
                  "path's FP64 polish included) with the device synchronised",
    }


def run_scf_leg(cell, looplimit):
    """The SCF half of the metric on the Si512 cell of the sweep: kukan's SCF
    (the dataset's local pseudopotential, Broyden mixing, RR + DIIS every
    iteration, Hartree CG, PZ LDA, Fermi-Dirac occupations for 2048 electrons
    in 1100 bands), mixed against plain FP64."""
    out = {"workload": "Si512 SCF: 128^3 grid, 1100 bands (2048 electrons, Fermi-Dirac kT "
                       "3e-3 Ha), Si PAW projectors with the dataset's D and S (no one-centre "
                       "update), the dataset's local pseudopotential (pseudocalc soft + hard "
                       f"parts), seeded smooth random start bands, Broyden mixing (eta {SCF_ETA},"
                       f" {SCF_NBRYDN} steps), RR + DIIS every iteration, Hartree CG (epsvh "
                       "1e-12, at most 800 iterations) on the 256^3 dense grid"}
    out.update(run_scf_pair(cell, NB, 1024, looplimit, ncgscf=0))
    return out


def run_scf_si64(looplimit):
    """The same comparison on the Si64 PAW cell (2x2x2 diamond, a = 20.52 bohr,
    64^3 grid, 160 bands for 256 electrons, atoms displaced by sigma = 0.05
    bohr from seed 1, DIIS after 3 CG steps)."""
    from rspacedist_b200 import system as S
    ds = S.load_dataset("si_paw")
    cell = S.make_cell(2 * A_SI, 64, S.diamond_positions(2, A_SI, 0.05, 1), ds)
    out = {"workload": "Si64 SCF: 64^3 grid, 160 bands (256 electrons, Fermi-Dirac kT 3e-3 Ha),"
                       " sigma 0.05 bohr seed 1, Si PAW projectors with the dataset's D and S, "
                       "the dataset's local pseudopotential, seeded smooth random start bands, "
                       f"Broyden (eta {SCF_ETA}, {SCF_NBRYDN} steps), 3 CG steps then RR + DIIS,"
                       " Hartree CG on the 128^3 dense grid"}
    out.update(run_scf_pair(cell, 160, 128, looplimit, ncgscf=3))
    return out


def run_force_check(ncomp=6, step=1e-3):
    """Forces of the Si64 PAW cell (2x2x2 diamond, a = 20.52 bohr, 64^3 grid,
    160 bands, atoms displaced by sigma = 0.10 bohr from seed 3) by the
    adjoint pass after a converged FP64 and mixed SCF (3 CG steps, then RR +
    DIIS, from seeded smooth random bands): against minus the
    central difference of the SCF free energy over +-step bohr on `ncomp`
    atom-axis components drawn from seed 3, and the projector part against
    force_eig_r (finite-difference band derivatives).  Prints one JSON line."""
    import torch
    from rspacedist_b200 import forces, kukan as K, lib, scf, system as S
    ds = S.load_dataset("si_paw")
    pos0 = S.diamond_positions(2, A_SI, 0.10, 3)
    mk = lambda p: S.make_cell(2 * A_SI, 64, p, ds)
    prm = lib.solver_prm(ncgscf=3)
    # every SCF from the same seeded smooth random bands (the ground state; see
    # run_scf), converged until the free energy moves by less than 1e-10
    # Ha/atom per iteration, so the energy differences resolve 1e-6 Ha/bohr
    # (the mixed SCF only gives forces: it stops at diff_charge < 1e-7 and the
    # SCF legs' energy bound, as FP32 bands resolve neither 1e-8 nor 1e-10)
    run = lambda c, dt: scf.run_scf(c, 160, 128, dtype=dt, prm=prm, eta=SCF_ETA,
                                    nbrydn=SCF_NBRYDN,
                                    eps_scf=1e-8 if dt == torch.float64 else 1e-7,
                                    eps_energy=1e-10 if dt == torch.float64 else SCF_EPS_ENERGY,
                                    looplimit=600, start="random", seed=0)
    cell = mk(pos0)
    out = {"force_check": {"cell": "Si64 PAW 64^3, 160 bands, sigma 0.10 seed 3",
                           "step_bohr": step}}
    t = time.perf_counter()
    r64 = run(cell, torch.float64)
    f64 = forces.atomic_forces(cell, r64)
    out["fp64_scf"] = {"converged": r64.converged, "iterations": r64.iterations,
                       "seconds": round(r64.seconds, 2)}
    r32 = run(cell, torch.float32)
    f32 = forces.atomic_forces(cell, r32)
    out["mixed_scf"] = {"converged": r32.converged, "iterations": r32.iterations,
                        "seconds": round(r32.seconds, 2)}
    out["max_abs_force_diff_mixed_vs_fp64"] = float(np.abs(f32["total"] - f64["total"]).max())
    g = K.Geometry(cell)
    dij = torch.tensor(cell.dij, dtype=torch.float64, device="cuda")
    sss = torch.tensor(cell.sss, dtype=torch.float64, device="cuda")
    fe = K.force_eig(g, dij, sss, r64.bands.psi, torch.tensor(r64.sval, device="cuda"),
                     torch.tensor(r64.occ, device="cuda")).cpu().numpy()
    out["max_abs_diff_projector_vs_force_eig"] = float(np.abs(f64["projector"] - fe).max())
    out["max_abs_force"] = float(np.abs(f64["total"]).max())
    rng = np.random.default_rng(3)
    comps = [(int(rng.integers(cell.natom)), int(rng.integers(3))) for _ in range(ncomp)]
    rows = []
    for a, ax in comps:
        es = []
        for sgn in (1, -1):
            p = pos0.copy()
            p[a, ax] += sgn * step
            es.append(run(mk(p), torch.float64).energy["free"])
        fd = -(es[0] - es[1]) / (2 * step)
        rows.append({"atom": a, "axis": ax, "adjoint": float(f64["total"][a, ax]), "fd": fd,
                     "diff": float(f64["total"][a, ax] - fd)})
    out["fd_components"] = rows
    out["max_abs_diff_adjoint_vs_fd"] = max(abs(x["diff"]) for x in rows)
    out["seconds"] = round(time.perf_counter() - t, 1)
    print(json.dumps(out), flush=True)


def host_bytes_available() -> int:
    """MemAvailable of this host in bytes (0 when unknown)."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def cpu_sample(cell, nthreads=None, nbands=CPU_SAMPLE_BANDS):
    """Inputs of one bounded sample of the sweep on the host cores:
    `nbands` seeded FP64 bands of the Si512 cell, their stored <p|psi>
    (computed before any clock starts, as the GPU sweep also takes them as
    input) and the oracle's system; run_cpu_sample times it."""
    from oracle import oracle as O
    from rspacedist_b200 import system as S
    nthreads = nthreads or os.cpu_count()
    if nbands is None:
        nbands = max(4, min(64, nthreads))
    geo = dict(natom=cell.natom, nprjmx=cell.nprjmx, num_list=cell.num_list, nprj=cell.nprj,
               natinf=cell.natinf, lst=cell.lst, v=cell.vnlocp.ravel())
    veff = S.smooth_veff(cell, 1)
    sysk = O.make_sys(geo, cell.shape, 4, cell.h, veff, cell.dij, cell.sss)
    psi = np.random.default_rng(0).standard_normal((nbands, cell.N)) * 0.1
    rp = O.nl_dot(geo, psi, cell.N).reshape(nbands, cell.natom, cell.nprjmx)
    O.hpsi_fast(sysk, psi[:1], rp[:1], 1)
    sample = {"nbands": nbands, "threads": nthreads, "psi": psi, "rp": rp, "veff": veff,
              "sys": sysk}
    run_cpu_sample(sample)
    return sample


def run_cpu_sample(sample):
    """The oracle's FP64 H psi (kukan's loops, bands spread over the host
    threads) of the sample; its wall time goes into sample['seconds']."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    sample["hpsi"] = O.hpsi_fast(sample["sys"], sample["psi"], sample["rp"], sample["threads"])
    sample["seconds"] = time.perf_counter() - t0
    return sample["seconds"]


def cpu_baseline(cell, sample):
    """GB/s of the oracle sample: the algorithmic bytes of an H psi call on
    the sample's bands (the same formula as the GPU value) over its time."""
    entries = int(sum(int(n) for n in cell.natinf))
    byts = algorithmic_bytes(cell, sample["nbands"], entries)
    return {"value": round(byts / sample["seconds"] / 1e9, 3), "unit": "GB/s",
            "cores": sample["threads"], "kind": "port",
            "sample": f"{sample['nbands']} of {NB} bands of the Si512 sweep (FP64 oracle H*psi "
                      f"with stored <p|psi>, {sample['seconds']:.2f} s on "
                      f"{sample['threads']} threads)",
            "band_points_per_s": round(sample["nbands"] * cell.N / sample["seconds"], 1)}


def check_parity(cell, g, dij, sample):
    """The GPU H psi of the CPU sample's bands against the oracle's output:
    <p|psi> and H psi on the FP64 path (bit for bit), H psi on the FP32 path
    (largest difference relative to max |H psi|)."""
    import torch
    from rspacedist_b200 import kukan as K
    dev = torch.device("cuda")
    psi64 = torch.tensor(sample["psi"], device=dev)
    rp_ref = sample["rp"]
    rp_gpu = K.nonlocaloperation_01(g, psi64).cpu().numpy()
    rp_t = torch.tensor(rp_ref, device=dev)
    h64 = K.hpsi(g, torch.tensor(sample["veff"], device=dev), dij, rp_t, psi64).cpu().numpy()
    h32 = K.hpsi(g, torch.tensor(sample["veff"], dtype=torch.float32, device=dev), dij, rp_t,
                 psi64.float()).cpu().numpy()
    ref = sample["hpsi"]
    scale = float(np.abs(ref).max())
    return {"bands": sample["nbands"], "against": "CPU oracle (FP64 restatement of "
            "kslaplacian_r + nonlocaloperation_r_01/_02) on the sampled bands",
            "nl_dot_f64_bitexact": bool(np.array_equal(rp_gpu, rp_ref)),
            "hpsi_f64_bitexact": bool(np.array_equal(h64, ref)),
            "max_abs_err_f64": float(np.abs(h64 - ref).max()),
            "max_rel_err_f32": float(np.abs(h32 - ref).max() / scale)}


def run_reference(args):
    """The CPU arm: every step is one bounded sample of the Si512 sweep run by
    the oracle on all host threads (set-up, lists included, by the oracle:
    the CUDA library is never loaded).  ms_per_step is the sample's measured
    time and value its algorithmic bytes over that time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cell = make_cell(list_builder=oracle_lists)
    sample = cpu_sample(cell)
    for _ in range(args.warmup):
        run_cpu_sample(sample)
    secs = [run_cpu_sample(sample) for _ in range(args.steps)]
    nbands, cores = sample["nbands"], sample["threads"]
    entries = int(sum(int(n) for n in cell.natinf))
    byts = algorithmic_bytes(cell, nbands, entries)
    v = byts * len(secs) / sum(secs) / 1e9
    print(json.dumps({
        "impl": "reference",
        "metric": "Si512 H*psi sweep HBM GB/s (FP32 psi); SCF time to eps in 'scf'",
        "value": round(v, 3), "unit": "GB/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(statistics.mean(secs) * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Si512 geometry, random psi, synthetic smooth veff)",
        "config": {"workload": "Si512 H*psi sweep: 128^3 grid, 1100 bands, 512 Si atoms x 12 "
                               "projectors; each step a sample of "
                               f"{nbands} bands on the CPU oracle (FP64 restatement of "
                               "kukan's loops)", "bands_per_step": nbands},
        "band_points_per_s": round(nbands * cell.N * len(secs) / sum(secs), 1),
        "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": cores, "kind": "port",
                         "sample": f"{nbands} of {NB} bands per step (FP64 oracle H*psi with "
                                   "stored <p|psi>)"},
        "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_diag_profile(dtype_name, which="si512"):
    """One scf_diag call (RR + DIIS) on the Si512 cell with 1100 smooth start
    bands (or the Si64 cell with 160) and the cell's local pseudopotential as
    the potential, run once to warm the memory pool and once more between
    cudaProfilerStart/Stop, so that `ncu --profile-from-start off` lists the
    kernels of exactly one call.  Prints the wall time of the profiled call."""
    import torch
    from rspacedist_b200 import kukan as K, lib, scf, system as S
    if which == "si64":
        cell = S.make_cell(2 * A_SI, 64, S.diamond_positions(2, A_SI, 0.05, 1),
                           S.load_dataset("si_paw"))
        nbands = 160
    else:
        cell = make_cell()
        nbands = NB
    g = K.Geometry(cell)
    dt = torch.float32 if dtype_name == "f32" else torch.float64
    from rspacedist_b200 import pseudo
    veff = pseudo.local_potential(cell)[0].to(dt)
    dij = torch.tensor(cell.dij, device="cuda")
    sss = torch.tensor(cell.sss, device="cuda")
    b = K.Bands(g, scf.smooth_start_bands_device(cell.shape, nbands, 0, dt), sss)
    K.orthogonalization(b, 1)
    prm = lib.solver_prm(ncgscf=0)
    K.scf_diag(b, veff, dij, 1, prm)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    t = time.perf_counter()
    K.scf_diag(b, veff, dij, 2, prm)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    print(json.dumps({"scf_diag": dtype_name, "seconds": round(time.perf_counter() - t, 4),
                      "bands": nbands, "grid": list(cell.shape)}), flush=True)


def run_proj_profile(npmesh, sample):
    """Projector-table generation (rs_projector_tables: Fourier-filtered
    projectors on the npmesh fine mesh and the double-grid contraction of
    pseudocalc_07) for the 512 atoms of the Si512 cell: one warm call, then
    three timed calls on the wall clock (host lists in, host vnlocp out), and
    the oracle on `sample` atoms scaled to 512.  Prints one JSON line with the
    largest difference from the oracle over the sampled atoms."""
    import torch
    from oracle import oracle as O
    from rspacedist_b200 import projectors as PR
    cell = make_cell()
    PR.projector_tables(cell, npmesh=npmesh)
    torch.cuda.synchronize()
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        v = PR.projector_tables(cell, npmesh=npmesh)
        ts.append(time.perf_counter() - t)
    # the same tables left in device memory, timed with CUDA events on the
    # launching stream (list upload and kernels; no copy back)
    vd = torch.empty(v.shape, dtype=torch.float64, device="cuda")
    PR.projector_tables(cell, npmesh=npmesh, out=vd)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tds = []
    for _ in range(3):
        e0.record()
        PR.projector_tables(cell, npmesh=npmesh, out=vd)
        e1.record()
        torch.cuda.synchronize()
        tds.append(e0.elapsed_time(e1) / 1e3)
    assert np.array_equal(vd.cpu().numpy(), v)
    ds = cell.ds
    coef, nqct, nqmx = PR.bessel_coefs(ds, cell.h)
    col, ym = PR.channel_table(ds)
    L = cell.num_list
    sl = lambda a: np.ascontiguousarray(a[:sample * L])
    lists = dict(natx=cell.natxyz[0][:sample], naty=cell.natxyz[1][:sample],
                 natz=cell.natxyz[2][:sample], natinf=cell.natinf[:sample],
                 lstx=sl(cell.lstxyz[0]), lsty=sl(cell.lstxyz[1]), lstz=sl(cell.lstxyz[2]))
    t = time.perf_counter()
    ref = O.projector_tables(cell.atoms[:sample], lists, cell.nmax, cell.h, cell.npmax, 4, npmesh,
                             L, col, ym, coef, nqct, nqmx, ds["rcut"], PR.PSFTRAD, PR.PSCTOFF,
                             PR.EPS, PR.NFILTYP, PR.FILPP, O.dg_weights(4, npmesh))
    tc = (time.perf_counter() - t) * cell.natom / sample
    err = float(np.abs(v[:sample] - ref).max() / np.abs(ref).max())
    print(json.dumps({"proj_profile": {"atoms": cell.natom, "projectors": len(col), "npmesh": npmesh,
                                       "nqct": nqct, "num_list": L},
                      "gpu_s": [round(x, 4) for x in ts],
                      "gpu_device_out_s": [round(x, 4) for x in tds],
                      "oracle_s_scaled": round(tc, 2), "oracle_sample_atoms": sample,
                      "oracle_threads": 1, "max_rel_diff": err}), flush=True)


def run_gemm_profile(npts):
    """The subspace contractions of the Rayleigh-Ritz step at the Si512 band
    count: Psi^T H Psi (rs_gram_f32, 1100 x 1100 over npts points) and the
    rotation Psi Z (rs_rotate_f32), random FP32 operands, each timed with CUDA
    events after one warm call; the error is against FP64 torch products.
    Prints one JSON line; the flop counts are the algorithmic 2 M^2 npts."""
    import ctypes as C
    import torch
    from rspacedist_b200 import lib
    lib.load()
    M = NB
    p = lambda t: C.c_void_p(t.data_ptr())
    s = lambda: C.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    A = torch.randn((M, npts), generator=g, device="cuda", dtype=torch.float32)
    B = torch.randn((M, npts), generator=g, device="cuda", dtype=torch.float32)
    G = torch.empty((M, M), dtype=torch.float64, device="cuda")
    Z = torch.randn((M, M), generator=g, device="cuda", dtype=torch.float64) / M ** 0.5
    Y = torch.empty((M, npts), dtype=torch.float32, device="cuda")

    def ev(fn, n=3):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    flop = 2.0 * M * M * npts
    out = {"gemm_profile": {"bands": M, "points": npts}}
    tg = ev(lambda: lib.call("rs_gram_f32", M, M, npts, p(A), npts, p(B), npts, 1.0, p(G), M,
                             0, s()))
    ref = (A.double() @ B.double().T).T
    out["gram_ms"] = round(tg, 3)
    out["gram_tflops"] = round(flop / tg / 1e9, 1)
    out["gram_rel_err"] = float((G - ref).abs().max() / ref.abs().max())
    del ref
    tr = ev(lambda: lib.call("rs_rotate_f32", npts, M, M, p(A), npts, p(Z), M, p(Y), npts, s()))
    ref = Z @ A.double()
    out["rotate_ms"] = round(tr, 3)
    out["rotate_tflops"] = round(flop / tr / 1e9, 1)
    out["rotate_rel_err"] = float((Y.double() - ref).abs().max() / ref.abs().max())
    print(json.dumps(out), flush=True)


def run_hartree_profile(n, mixed=False):
    """The Hartree CG Poisson solve (rs_hartree_cg, nfh = 4, epsvh = 1e-12, at
    most 800 iterations) on an n^3 grid of the Si512 cell (a = 41.04 bohr):
    eight normalised Gaussians (sigma = 1 bohr, centres uniform in the cell
    from seed 0) on a uniform neutralising background, as in the reference's
    standalone Hartree test.  One 50-iteration warm call, then one solve from
    zero timed on the wall clock with the device synchronised, both on one side
    stream; prints one JSON
    line with the per-iteration time and 88 B/pt/iteration bandwidth."""
    import torch
    from rspacedist_b200 import kukan as K
    a = 4 * 10.26
    h = a / n
    x = (np.arange(n) + 0.5) * h - a / 2
    rng = np.random.default_rng(0)
    rho = np.zeros((n, n, n))
    sig = 1.0
    for c in rng.uniform(-a / 2, a / 2, (8, 3)):
        d = [x - c[k] for k in range(3)]
        d = [di - a * np.round(di / a) for di in d]
        r2 = d[2][:, None, None] ** 2 + d[1][None, :, None] ** 2 + d[0][None, None, :] ** 2
        rho += np.exp(-r2 / (2 * sig * sig)) / (2 * np.pi * sig * sig) ** 1.5
    rho -= rho.mean()
    rho_d = torch.tensor(rho.ravel(), device="cuda")
    vh = torch.zeros_like(rho_d)
    xm = (a / 2,) * 3
    side = torch.cuda.Stream()  # a real stream: the solve replays its batches as a graph
    # the warm call on the same stream, so that the timed solve finds its work
    # vectors in the stream's memory pool
    with torch.cuda.stream(side):
        K.scf_hartree((n, n, n), 4, xm, rho_d, vh, 1e-12, ncgmax=50, mixed=mixed)
    torch.cuda.synchronize()
    vh.zero_()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk, torch.cuda.stream(side):
        t = time.perf_counter()
        it, dp = K.scf_hartree((n, n, n), 4, xm, rho_d, vh, 1e-12, mixed=mixed)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
    print(json.dumps({"hartree_profile": {"grid": [n] * 3, "cell_bohr": a,
                                          "solve": "mixed (FP32 vectors)" if mixed else "FP64"},
                      "iterations": it,
                      "dp": dp, "ms": round(dt * 1e3, 2), "clocks": clk.summary(),
                      "us_per_iter": round(dt / it * 1e6, 1),
                      "gbs_at_88_bytes_per_point": round(88 * n ** 3 / (dt / it) / 1e9, 1)}),
          flush=True)


def run_batch_profile(ncell, nbands):
    """H psi of a set of small independent cells (16 Si8 + 16 C8 by default,
    20 bands each, grids 22^3-36^3): a loop of single-cell rs_hpsi_f32 calls
    against one persistent rs_hpsi_batch launch, direct and as a CUDA graph
    replay, each timed with CUDA events on a side stream over 20 repetitions.
    Prints one JSON line."""
    import torch
    from rspacedist_b200 import kukan as K, system as S
    cells = S.small_cell_set(ncell)
    geoms = [K.Geometry(c) for c in cells]
    veff = [torch.tensor(S.smooth_veff(c, i), dtype=torch.float32, device="cuda")
            for i, c in enumerate(cells)]
    dij = [torch.tensor(c.dij, dtype=torch.float64, device="cuda") for c in cells]
    psi = [torch.tensor(S.random_bands(c, nbands, i), dtype=torch.float32, device="cuda")
           for i, c in enumerate(cells)]
    rp = [K.nonlocaloperation_01(g, p) for g, p in zip(geoms, psi)]
    out = [torch.empty_like(p) for p in psi]
    plan = K.HpsiBatch(geoms, [nbands] * ncell)
    plan.set(veff, dij, rp, psi, out)
    st = torch.cuda.Stream()
    reps = 20

    def timed(fn):
        with torch.cuda.stream(st):
            for _ in range(3):
                fn()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            for _ in range(reps):
                fn()
            b.record(st)
        st.synchronize()
        return a.elapsed_time(b) / reps

    def loop():
        for g, v, d, r, p, o in zip(geoms, veff, dij, rp, psi, out):
            K.hpsi(g, v, d, r, p, out=o)

    t_loop = timed(loop)
    t_batch = timed(lambda: plan.run(graph=False))
    t_graph = timed(lambda: plan.run(graph=True))
    tuned = plan.info()
    pts = sum(c.N for c in cells) * nbands
    # every candidate form, fixed in turn (the same bits; the autotuner's pick is above)
    shapes = {}
    for sh in [(128, 4, 8), (256, 4, 4), (256, 8, 4), (64, 2, 16)]:
        plan.set_shape(*sh)
        shapes["%d/%d/%d" % sh] = round(timed(lambda: plan.run(graph=False)), 4)
    print(json.dumps({"batch_profile": {"cells": ncell, "bands": nbands,
                                        "grids": sorted({c.shape[0] for c in cells}),
                                        "band_points": pts},
                      "per_cell_calls_ms": round(t_loop, 4), "batched_ms": round(t_batch, 4),
                      "batched_graph_ms": round(t_graph, 4),
                      "speedup_graph_vs_calls": round(t_loop / t_graph, 2),
                      "autotuned": tuned, "fixed_shapes_ms": shapes}), flush=True)
    plan.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-fp64-sweep", dest="fp64_sweep", action="store_false",
                    help="skip the plain FP64 sweep")
    ap.add_argument("--profile-range", choices=["sweep", "stencil"],
                    help="bracket the timed sweep steps (sweep) or the timed stencil-only "
                         "launches (stencil) with cudaProfilerStart/Stop, for ncu "
                         "--profile-from-start off")
    ap.add_argument("--staging", choices=["tma", "cp"], default="tma",
                    help="plane staging of the FP32 stencil: tensor-map loads or cp.async")
    ap.add_argument("--bands", type=int, default=NB,
                    help="bands per sweep (default 1100; smaller values for profiling only)")
    ap.add_argument("--scf-loops", "--scf-iters", dest="scf_loops", type=int, default=300,
                    help="iteration limit of the Si512 SCF run per path (0 skips the leg)")
    ap.add_argument("--force-check", action="store_true",
                    help="run the Si64 force check (adjoint vs energy differences) and exit")
    ap.add_argument("--force-step", type=float, default=1e-3,
                    help="with --force-check: the finite-difference step in bohr")
    ap.add_argument("--diag-profile", choices=["f32", "f64"],
                    help="run one profiled scf_diag call of the SCF leg and exit")
    ap.add_argument("--diag-cell", choices=["si512", "si64"], default="si512",
                    help="with --diag-profile: the cell (Si512 with 1100 bands, Si64 with 160)")
    ap.add_argument("--gemm-profile", type=int, metavar="POINTS",
                    help="time the tensor-core Gram and rotation at 1100 bands x POINTS and exit")
    ap.add_argument("--hartree-profile", type=int, metavar="N",
                    help="time the Hartree CG solve on an N^3 dense grid and exit")
    ap.add_argument("--mixed", action="store_true",
                    help="with --hartree-profile: the mixed-precision solve")
    ap.add_argument("--proj-profile", type=int, metavar="NPMESH",
                    help="time the projector-table generation of the Si512 cell and exit")
    ap.add_argument("--batch-profile", type=int, metavar="CELLS",
                    help="time H*psi of CELLS small cells, per-cell calls vs one batched "
                         "launch, and exit")
    args = ap.parse_args()
    if args.force_check:
        run_force_check(step=args.force_step)
    elif args.proj_profile:
        run_proj_profile(args.proj_profile, 4)
    elif args.batch_profile:
        run_batch_profile(args.batch_profile, 20)
    elif args.hartree_profile:
        run_hartree_profile(args.hartree_profile, args.mixed)
    elif args.diag_profile:
        run_diag_profile(args.diag_profile, args.diag_cell)
    elif args.gemm_profile:
        run_gemm_profile(args.gemm_profile)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
