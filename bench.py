#!/usr/bin/env python
"""Benchmark: Yee cell-updates/s of the 3D CPML time-stepping hot path.

Workload: 3D TM planar waveguide 480 x 192 x 256 cells @ 30 nm,
float32 fields, 10-cell CPML, absorbing aqueous (1.333+0.001i), two seeded
polystyrene beads, 4000-step CW schedule with Ex/Ey/Ez phasors.  One "step" is
one leapfrog time step over the whole grid.  The K timed steps sample the
schedule in its own proportions: steps outside the 8-period DFT window and
steps inside it (detector boxes every step, |E|^2 averaging at its cadence).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one per GPU, launched by torchrun): the path
has no exchange step, so there is no collective in the data path; the timing is
the max over ranks.  --impl reference times the reference algorithm's CPU
implementation (the NumPy oracle restatement of the reference path; the
reference package itself is pure NumPy/CuPy Python and is not installed on the
GPU machine).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = 'yee_cell_updates_per_s'
UNIT = 'cell-updates/s'
WORKLOAD = ('waveguide3d_tm: 3D TM planar waveguide 480x192x256 @ 30 nm, fp32, 10-cell CPML, '
            'lossy aqueous 1.333+0.001i, 2 seeded PS beads, 4000-step CW schedule, Ex/Ey/Ez phasors')


def dist_env():
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    return ws, int(os.environ.get('RANK', '0')), int(os.environ.get('LOCAL_RANK', '0'))


def max_over_ranks(x, pg, device='cuda'):
    """The slowest rank's figure (every rank must call it, in the same order);
    x itself without a process group."""
    if not pg:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_rate(cells, steps, ws, seconds):
    """Whole-job cell updates per second: ws replicas, each `steps` steps of `cells`."""
    return cells * steps * ws / seconds


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class Clocks:
    """nvidia-smi sampler of SM clock and throttle reasons during a region."""
    Q = ('timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, dev_uuid=None):
        cmd = ['nvidia-smi', '--query-gpu=' + self.Q, '--format=csv,noheader,nounits', '-lms', '100']
        if dev_uuid:
            cmd.insert(1, '--id=' + dev_uuid)
        try:
            self.p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=10)
        except Exception:
            self.p.kill()
            out = ''
        rows = [[c.strip() for c in ln.split(',')] for ln in out.splitlines() if ln.count(',') >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace('.', '').isdigit()]
        load = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == 'active'})
        return dict(sm_mhz=statistics.median(load) if load else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(rows))


def split_steps(K, steps_total, n_acc):
    """K timed steps split in the schedule's proportions (outside / inside the DFT window)."""
    kb = int(round(K * n_acc / steps_total))
    return K - kb, kb


def cpu_baseline(spec, steps=16, warmup=1):
    """The NumPy oracle (restatement of the reference path) on a bounded sample:
    `steps` consecutive full-grid steps with the detector sums, one host thread,
    after `warmup` untimed steps."""
    from oracle import harness as H
    from oracle import fdtd_oracle as O
    c = oracle_case(spec)
    s = H.setup_3d(c)
    g = O.Grid3D(spec.nx, spec.ny, spec.nz, s['dx'], s['dt'], s['cpml'], (s['ce_x'], s['ce_y'], s['ce_z']),
                 s['da'], s['src'], 'Ey' if spec.pol == 'p' else 'Ez')
    nsp = s['n_sp']
    box = (slice(64, 130), slice(100, 167), slice(nsp, spec.nz - nsp))
    for n in range(max(1, warmup)):
        g.step(n, 0.0)
    t0 = time.perf_counter()
    for n in range(max(1, warmup), max(1, warmup) + steps):
        g.step(n, 0.5)
        g.box_e2(*box)
    dt = time.perf_counter() - t0
    cells = spec.nx * spec.ny * spec.nz
    return cells * steps / dt, dict(sample=f'{steps} consecutive full-grid steps of the 480x192x256 3D CPML '
                                           f'step + detector box sums on the NumPy oracle (float32), '
                                           f'{dt:.1f} s', cores=1)


def oracle_case(spec):
    st = spec.stack
    return dict(pol=spec.pol, Nx=spec.nx, Ny=spec.ny, Nz=spec.nz, dx_nm=spec.dx_nm, t_wg_um=st.t_wg_um,
                tear_um=spec.tear_um, stack=[[t, [complex(n).real, complex(n).imag]] for t, n in st.layers],
                n_sub=st.n_sub, wg_n=st.wg_n, npml=spec.npml, lam_nm=spec.lam_nm, waist_um=spec.waist_um,
                beads=[dict(x_um=b.x_um, d_um=b.d_um, n=b.n, y_um=b.y_um, z_um=b.z_um) for b in spec.beads])


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from lens_sensor_b200.workloads import waveguide3d_tm
    spec, steps_total = waveguide3d_tm()
    # each step: one full-grid oracle step; bounded so the arm ends within minutes
    k = max(1, min(args.steps, 12))
    w = max(1, min(args.warmup, 10))
    value, info = cpu_baseline(spec, steps=k, warmup=w)
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=ws, steps=k, warmup=w,
                ms_per_step=spec.nx * spec.ny * spec.nz / value * 1e3, higher_is_better=True,
                scaling='weak', vs_baseline=None, dtype='f32', data='synthetic',
                config=dict(workload=WORKLOAD, cells=spec.nx * spec.ny * spec.nz, steps_total=steps_total),
                impl='reference', cpu_baseline=dict(value=value, unit=UNIT, cores=info['cores'], kind='port',
                                                   sample=info['sample']),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def run_e2e(spec, steps_total, cells, ws, pg, engine='fused'):
    """The whole solve through the public API from host inputs: host setup,
    upload, the 4000-step schedule, read-back of the three phasors."""
    import torch
    from lens_sensor_b200.solver3d import Solve3D
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2 = Solve3D(spec, steps_total, comps=(0, 1, 2), engine=engine)
    torch.cuda.synchronize()          # the uploads are synchronous already; marks the phase end
    t1 = time.perf_counter()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    s2.stage_host((0, 1, 2))          # the read-back's host buffers are made while the device steps
    s2.run()
    ev[1].record()
    ph = s2.phasors_host((0, 1, 2))
    res = s2.results()
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    t_e2e = max_over_ranks(t3 - t0, pg)
    d2h = s2.d2h_bytes + 64
    t_run = ev[0].elapsed_time(ev[1]) * 1e-3
    phases = dict(setup_host=s2.t_setup_host, setup_device=t1 - t0 - s2.t_setup_host, run_device=t_run,
                  after_run=t3 - t1 - t_run)
    out = dict(value=job_rate(cells, steps_total, ws, t_e2e), unit=UNIT, h2d_bytes_per_step=s2.h2d_bytes / steps_total,
               d2h_bytes_per_step=d2h / steps_total, solve_seconds=t_e2e, host_setup_seconds=s2.t_setup_host,
               phase_seconds={k: round(v, 4) for k, v in phases.items()},
               transmission=res['transmission'], cw_rel_change=res['cw_rel_change'])
    out['err_vs_fp64'] = err3d_vs_fp64(spec, ph, res, s2)
    del s2
    torch.cuda.empty_cache()
    return out


FP64 = os.path.join(ROOT, 'tests', 'golden', 'fp64')


def _fp64_meta():
    try:
        with open(os.path.join(FP64, 'fp64.json')) as f:
            return json.load(f)['runs']
    except Exception:
        return None


def _sample_mask(n, shift):
    """The fixtures' hashed cell sample (tests/golden/make_fp64.py sample_mask)."""
    i = np.arange(n, dtype=np.uint64)
    return (((i * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) >> np.uint64(32 - shift)) == 0


def _rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def err3d_vs_fp64(spec, ph, res, solve):
    """Relative L2 errors of the config-1 phasors (hashed 1/256 cell sample and z
    mid-plane; Ex, Ez against the vector norm) and scalars against the FP64 run
    of the reference algorithm (tests/golden/fp64), with the reference
    algorithm's own float32 errors beside them."""
    m = _fp64_meta()
    if m is None or 'c1' not in m:
        return None
    fx = np.load(os.path.join(FP64, 'c1.npz'))
    r = m['c1']
    vs = np.sqrt(sum(np.linalg.norm(fx[f'{k}_sample']) ** 2 for k in ('Ex', 'Ey', 'Ez')))
    out = {}
    for q, c in enumerate(('Ex', 'Ey', 'Ez')):
        a = ph[q]
        sel = a.ravel()[_sample_mask(a.size, 8)]
        out[c] = dict(own=_rel(sel, fx[f'{c}_sample']), vector=float(np.linalg.norm(sel - fx[f'{c}_sample']) / vs),
                      zmid=_rel(a[:, :, a.shape[2] // 2], fx[f'{c}_zmid']))
    for k in ('P_in', 'P_out', 'transmission'):
        out[k] = abs(res[k] - r[k]) / max(abs(r[k]), 1e-300)
    out['bar'] = 1e-4
    out['reference_fp32'] = {c: r['ref_fp32_err'][c] for c in ('Ex', 'Ey', 'Ez', 'transmission')}
    return out


def cpu_baseline_2d(spec, steps=200):
    """The NumPy oracle (restatement of the reference 2D TE path) on `steps`
    consecutive full-grid steps, one host thread."""
    from oracle import fdtd_oracle as O
    from lens_sensor_b200.geometry import build_2d
    geo = build_2d(spec)
    src = O.Huygens.__new__(O.Huygens)
    src.ix, src.omega = int(geo['src']['ix']), float(geo['src']['omega'])
    src.amp, src.ph1, src.ph2 = (np.asarray(geo['src'][k], np.float32) for k in ('amp', 'ph1', 'ph2'))
    g = O.Grid2D('s', spec.nx, spec.ny, spec.dx, spec.dt, geo['cx'], geo['cy'], src,
                 {k: geo[k] for k in ('ce_e', 'ce_h')}, np.float32)
    g.step(0, 0.0)
    t0 = time.perf_counter()
    for n in range(1, steps + 1):
        g.step(n, 0.5)
    dt = time.perf_counter() - t0
    return spec.nx * spec.ny * steps / dt, f'{steps} consecutive full-grid steps of the 1600x480 2D TE CPML step ' \
                                            f'on the NumPy oracle (float32), {dt:.1f} s'


def run_planar2d(cpu=True):
    """Config 0 (planar2d_te: 2D TE 1600 x 480 @ 25 nm, 6000 steps, one-period CW
    phasor, Ez snapshots every 200 steps).  Each 2D engine runs the whole
    6000-step solve on the device (CUDA events, inputs resident; the batched and
    temporally blocked engines replay the schedule as one CUDA graph); value is
    the fastest engine's.  e2e: that engine's solve from the host spec (setup,
    upload, graph capture, run, read-back of the phasor and the 30 snapshots),
    the median of three whole solves."""
    import torch
    from lens_sensor_b200.solver2d import Solve2D
    from lens_sensor_b200.workloads import planar2d_te
    sp, steps = planar2d_te()
    cells = sp.nx * sp.ny
    geo = None
    rates = {}
    cands = [('resident', 0), ('batch', 2), ('batch', 4), ('batch', 8), ('persistent', 8), ('tb', 4), ('step', 4)]
    for eng, by in cands:
        warm = Solve2D(sp, steps, engine=eng, geo=geo, by=by)
        geo = warm.geo
        if eng in ('batch', 'tb'):
            warm.capture()
        warm.run()
        del warm
        s = Solve2D(sp, steps, engine=eng, geo=geo, by=by)
        if eng in ('batch', 'tb'):
            s.capture()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        s.run()
        ev[1].record()
        torch.cuda.synchronize()
        rates[(eng, by)] = (ev[0].elapsed_time(ev[1]) * 1e-3, s.launches)
        del s
    best_key = min(rates, key=lambda e: rates[e][0])
    best, best_by = best_key
    t_dev, launches = rates[best_key]
    t_all = []
    for rep in range(3):   # whole solves from the host spec; the median is reported
        if rep:
            del s
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s = Solve2D(sp, steps, engine=best, by=best_by)
        if best in ('batch', 'tb'):
            s.capture()
        s.stage_host()
        s.run()
        ph, snaps = s.host_results()
        t_all.append(time.perf_counter() - t0)
    t_e2e = float(np.median(t_all))
    peak, peak_src = peaks()
    achieved = 32.0 * cells / (t_dev / steps) / 1e9
    kern = {'resident': 'rs2d (one resident cooperative launch: the fields stay in registers for the whole '
                        'solve, bands of x rows exchange one row per half step through L2)',
            'batch': f'b2d_h + b2d_e (batched passes on one instance, tiles of 128 x {2 * best_by})',
            'persistent': 'pb2d (persistent cooperative launch)',
            'tb': 'tb2d (four steps per launch)', 'step': 'te2d_h + te2d_e (single-grid passes)'}[best]
    out = dict(workload=f'planar2d_te: 2D TE planar waveguide {sp.nx}x{sp.ny} @ 25 nm, fp32, 12-cell CPML, '
                        f'{steps} steps, CW ramped over 20 periods, one seeded PS bead, one-period phasor, '
                        'Ez snapshots every 200 steps',
               unit=UNIT, value=cells * steps / t_dev, ms_per_step=t_dev / steps * 1e3, steps=steps, cells=cells,
               engine=best, by=best_by,
               engines={f'{e}_by{b}': cells * steps / t for (e, b), (t, _) in rates.items()}, gpu_launches=launches,
               l2=f'working set {(5 * cells * 4) / 1e6:.0f} MB of fields and coefficients fits in the 126 MB L2: '
                  'the steps of one solve run L2-resident, as in use; no flush between steps',
               roofline=dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s', frac=achieved / peak,
                             peak_source=peak_src, kernel=kern, alg_bytes_per_step=32 * cells,
                             step_ms=t_dev / steps * 1e3,
                             note=('the resident launch moves no field bytes through HBM between its first and '
                                   'last step: achieved counts the 32 B per cell update of the HBM-streamed step, '
                                   'so frac > 1 is possible and means the on-chip engine beats the streamed bound')
                             if best == 'resident' else None),
               e2e=dict(value=cells * steps / t_e2e, unit=UNIT, solve_seconds=t_e2e,
                        solve_seconds_all=[round(t, 4) for t in t_all],
                        h2d_bytes_per_step=s.h2d_bytes / steps, d2h_bytes_per_step=s.d2h_bytes / steps,
                        host_setup_seconds=s.t_setup_host))
    m = _fp64_meta()
    if m and 'c0' in m:
        fx = np.load(os.path.join(FP64, 'c0.npz'))
        mk = _sample_mask(snaps[-1].size, 3)
        out['err_vs_fp64'] = dict(phasor=_rel(ph, fx['phasor']),
                                  snap_last=_rel(snaps[-1].ravel()[mk], fx['snap_last_sample']), bar=1e-4,
                                  reference_fp32=m['c0']['ref_fp32_err'])
    del s
    torch.cuda.empty_cache()
    if cpu:
        v, sample = cpu_baseline_2d(sp)
        out['cpu_baseline'] = dict(value=v, unit=UNIT, cores=1, kind='port', sample=sample)
    return out


def run_batched(plain_sample=16, count=256):
    """The sweep2d workload: 256 uneven 2D TE/TM solves (4000 steps each).

    plain   instances one at a time through the single-grid engine (the drop-in
            run_beads path, lens_te2d_step / lens_tm2d_step), on a seeded sample of
            `plain_sample` instances spread over the sweep;
    batched the whole sweep through batch2d.Sweep (autotuned tile and group
            budget, one CUDA graph per group), FP32 storage, then FP16 storage
            with each instance's phasor error against the FP32 run.
    Throughput is cell-updates/s over the whole timed region (device events)."""
    import torch
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200 import engine as E
    from lens_sensor_b200.workloads import sweep2d
    specs, steps = sweep2d(count=count)
    ev = lambda: torch.cuda.Event(enable_timing=True)
    sw = B.Sweep(specs, steps, 'f32')
    tuned = sw.autotune()
    for g in sw.groups:
        g.capture(sw.table)
    e0, e1 = ev(), ev()
    e0.record()
    launches = sw.run()
    e1.record()
    torch.cuda.synchronize()
    t_b = e0.elapsed_time(e1) * 1e-3
    cells = sw.cells()
    ref = [r['phasor'] for r in sw.results()]
    K = [r['K'] for r in sw.results()]
    idx = list(range(0, len(specs), max(1, len(specs) // plain_sample)))[:plain_sample]
    pc = 0
    e0.record()
    for q in idx:
        sp, geo = specs[q], sw.insts[q].geo
        coef = {k: geo[k] for k in ('ce_e', 'ce_h', 'ca_x', 'ca_y', 'da_x', 'da_y') if k in geo}
        g = E.Grid2D(sp.pol, sp.nx, sp.ny, sp.dx, sp.dt, coef, geo['cx'], geo['cy'], geo['src'])
        epi = E.Epi2D(g, dft=sw.insts[q].window)
        g.step(sw.table, 0, steps, epi)
        pc += sp.nx * sp.ny
    e1.record()
    torch.cuda.synchronize()
    t_p = e0.elapsed_time(e1) * 1e-3
    # the fastest one-at-a-time path: each sampled instance alone on the batched
    # kernels, its whole schedule replayed as one CUDA graph (Solve2D's 'batch' engine)
    t_g = 0.0
    for q in idx:
        one = B.Sweep([specs[q]], steps, 'f32', by=sw.by, geos=[sw.insts[q].geo])
        one.groups[0].capture(one.table)
        one.run()                      # the graph's first launch uploads it
        torch.cuda.synchronize()
        one.reset()
        e0.record()
        one.run()
        e1.record()
        torch.cuda.synchronize()
        t_g += e0.elapsed_time(e1) * 1e-3
        del one
    geos = [q.geo for q in sw.insts]
    by, budget = sw.by, sw.budget
    del sw
    torch.cuda.empty_cache()
    # the resident launches (lens_rs2d_run): the same instances one at a time, then
    # the whole sweep packed into launches that each hold as many as fit on the chip
    t_r1 = 0.0
    for q in idx:
        one = B.Sweep([specs[q]], steps, 'f32', geos=[geos[q]], resident=True)
        torch.cuda.synchronize()
        e0.record()
        one.run()
        e1.record()
        torch.cuda.synchronize()
        t_r1 += e0.elapsed_time(e1) * 1e-3
        del one
    sr = B.Sweep(specs, steps, 'f32', geos=geos, resident=True)
    sr.run()                               # warm-up (first launch of each plan)
    sr.reset()
    torch.cuda.synchronize()
    e0.record()
    sr.run()
    e1.record()
    torch.cuda.synchronize()
    t_res = e0.elapsed_time(e1) * 1e-3
    res_r = sr.results()
    res_err = []
    for q, r in enumerate(res_r):   # on the host: relative L2 difference, NaN where non-finite
        x, y = r['phasor'].cpu().numpy(), ref[q].cpu().numpy()
        res_err.append(float(np.linalg.norm((x - y).ravel()) / max(float(np.linalg.norm(y.ravel())), 1e-300)))
    res_groups = [dict(instances=len(g.insts), rows=g.rows, ctas=g.ctas, threads=g.threads) for g in sr.groups]
    res_ph = [r['phasor'] for r in res_r]
    del sr, res_r
    torch.cuda.empty_cache()
    sh = B.Sweep(specs, steps, 'f16', by=by, budget=budget, geos=geos)
    for g in sh.groups:
        g.capture(sh.table)
    e0.record()
    sh.run()
    e1.record()
    torch.cuda.synchronize()
    t_h = e0.elapsed_time(e1) * 1e-3
    res16 = sh.results()
    # the same FP32 sweep as one persistent cooperative launch per group (lens_batch2d_run)
    sp_ = B.Sweep(specs, steps, 'f32', by=by, budget=budget, geos=geos)
    e0.record()
    sp_.run(persistent=True)
    e1.record()
    torch.cuda.synchronize()
    t_pers = e0.elapsed_time(e1) * 1e-3
    pers_same = all(torch.equal(a['phasor'], b) for a, b in zip(sp_.results(), ref))
    del sp_
    err = [float((r['phasor'] - ref[q]).abs().norm() / max(float(ref[q].abs().norm()), 1e-300))
           for q, r in enumerate(res16)]
    fp64 = None
    m = _fp64_meta()
    if m:
        fp64 = dict(bar=1e-4)
        for q in [int(k[2:]) for k in m if k.startswith('sw') and int(k[2:]) < len(specs)]:
            fx = np.load(os.path.join(FP64, f'sw{q}.npz'))['phasor_sample']
            for tag, ph in (('f32', ref[q]), ('f16', res16[q]['phasor']), ('resident', res_ph[q])):
                a = ph.cpu().numpy()
                fp64[f'sw{q}_{tag}'] = _rel(a.ravel()[_sample_mask(a.size, 3)], fx)
    del sh
    torch.cuda.empty_cache()
    # the FP16 acceptance gate over the whole sweep (probes in both storages)
    e0.record()
    gres, gate = B.gated_sweep(specs, steps, 'f16', tol=1e-4, by=by, budget=budget, geos=geos)
    e1.record()
    torch.cuda.synchronize()
    t_gate = e0.elapsed_time(e1) * 1e-3
    gate['value'] = cells * steps / t_gate
    gate['probe_err_max'] = max(p['err'] for p in gate['probes'])
    del gres
    torch.cuda.empty_cache()
    plain = pc * steps / t_p
    plain_graph = pc * steps / t_g
    plain_resident = pc * steps / t_r1
    f32 = cells * steps / t_b
    f16 = cells * steps / t_h
    res = cells * steps / t_res
    return dict(workload=f'sweep2d: {len(specs)} uneven 2D TE/TM solves, widths 600-2400 x heights 300-560 @ 25 nm, '
                         '12-cell CPML, 4000 steps, seeded tear-film / lipid / bead sweep',
                unit=UNIT, cells_total=cells, steps=steps, plain=plain,
                plain_sample=f'{len(idx)} instances (every {len(specs) // len(idx)}th) one at a time, through '
                             'the drop-in single-grid engine (run_beads path)',
                plain_graph=plain_graph,
                plain_graph_sample='the same instances one at a time on the batched kernels, each schedule '
                                   'replayed as one CUDA graph (the fastest one-at-a-time path)',
                batched_f32=f32, batched_f16=f16, batched_vs_plain=f32 / plain, f16_vs_plain=f16 / plain,
                batched_vs_plain_graph=f32 / plain_graph,
                batched_persistent_f32=cells * steps / t_pers, persistent_identical_to_graphs=pers_same,
                plain_resident=plain_resident,
                plain_resident_sample='the same instances one at a time, each in one resident launch '
                                      '(lens_rs2d_run, fields in registers for the whole solve)',
                batched_resident_f32=res, resident_vs_plain=res / plain, resident_vs_plain_resident=res / plain_resident,
                resident_launches=res_groups, resident_phasor_err_vs_batched_f32_max=float(np.nanmax(res_err)),
                resident_phasor_nonfinite=int(np.sum(~np.isfinite(res_err))),
                tile=f'128 x {2 * by} nodes', group_budget_bytes=budget, autotune=tuned, graph_launches=launches,
                f16_phasor_err_vs_f32_max=max(err), f16_phasor_err_vs_f32_median=float(np.median(err)),
                K_median=float(np.median(K)), err_vs_fp64=fp64, f16_gate=gate)


def _stitch_member(pl, stream, pool):
    """One stitch job (a member of a sweep) on its own stream; the assembled
    slabs are written to host arrays."""
    from lens_sensor_b200 import engine as E
    from lens_sensor_b200.stitch3d import StitchSolve
    Ef = np.zeros((pl.Nx_full, pl.Nj, pl.Nk), np.complex64)
    Ia = np.zeros((pl.Nx_full, pl.Nj, pl.Nk), np.float32)

    def sink(w, g_lo, g_hi, Ew, I):
        Ef[g_lo:g_hi] = Ew
        Ia[g_lo:g_hi] = I
    return StitchSolve(pl, E, sink, stream=stream, pool=pool)


def stitch_vs_reference():
    """The reference's own characterization stitch (3 windows, the last flush;
    tests/golden/dropin_3d_stitch.json 'goldenstitch', from the reference's
    run_3d_stitched) through this drop-in on the GPU: relative errors of its
    result scalars and the |<E^2>| sum against the reference's values."""
    import tempfile
    from lens_sensor_b200 import fdtd3d_core as D3
    case = json.load(open(os.path.join(ROOT, 'tests', 'golden', 'dropin_3d_stitch.json')))['goldenstitch']
    cwd, kappa = os.getcwd(), D3.KAPPA
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            D3.KAPPA = dict(case['kappa'])
            r = D3.run_3d_stitched(**dict(case['kw']))
        finally:
            os.chdir(cwd)
            D3.KAPPA = kappa
    out = {k: abs(r[k] - case['result'][k]) / max(abs(case['result'][k]), 1e-300)
           for k in ('transmission', 'P_in', 'P_out')}
    out['case'] = 'reference characterization stitch: 3 windows, the last flush with the domain end'
    return out


def run_stitch(windows=3, members=2):
    """The stitch3d_plan workload: a 3D stitch of `windows` windows of 480 x 192 x
    256 cells (30 nm, 40-cell overlap; 19 windows = the whole 240 um guide) through
    stitch3d.StitchSolve: per-window geometry built on a host thread while the
    previous window runs, steady-state steps, on-device handoff of the overlap
    amplitudes, assembly to host memory.  Rate = cell updates of every window
    (absorber extension included) over the wall time from the first window's
    setup to the last window's assembled slab.  Then `members` independent
    members of a sweep (other seeds) run at once, each on its own CUDA stream,
    advanced in turn in quanta of steps, so one member's window setup, handoff
    and assembly overlap the others' steps."""
    import concurrent.futures as cf
    import torch
    from lens_sensor_b200.workloads import stitch3d_plan
    windows = 19 if windows <= 0 else windows
    nx_full = 480 + (windows - 1) * 440
    pl = stitch3d_plan(nx_full=nx_full)
    pool = cf.ThreadPoolExecutor(2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    job = _stitch_member(pl, None, pool)
    while not job.done:
        job.advance(pl.steps_win)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    cu = pl.cell_updates()
    T = job.transmission()
    del job
    torch.cuda.empty_cache()
    conc = None
    if members > 1:
        plans = [stitch3d_plan(seed=3 + 2 * q, nx_full=nx_full) for q in range(members)]
        streams = [torch.cuda.Stream() for _ in plans]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        jobs = [_stitch_member(p, s, pool) for p, s in zip(plans, streams)]
        while not all(j.done for j in jobs):
            for j in jobs:
                j.advance(256)
        torch.cuda.synchronize()
        wc = time.perf_counter() - t0
        cuc = sum(p.cell_updates() for p in plans)
        conc = dict(members=members, value=cuc / wc, wall_s=wc, cell_updates=cuc,
                    vs_one_member=(cuc / wc) / (cu / wall))
        del jobs
        torch.cuda.empty_cache()
    pool.shutdown()
    return dict(workload=f'stitch3d_plan: 3D stitch, {pl.n_win} windows of {pl.Nx_win} x {pl.Ny} x {pl.Nz} @ 30 nm '
                         f'(+{pl.EXT}-cell absorber on interior windows), {pl.O}-cell overlap, '
                         f'{pl.steps_win} steps per window; {pl.Nx_full} cells = {pl.lx_um:.1f} um',
                unit=UNIT, value=cu / wall, wall_s=wall, cell_updates=cu, windows=pl.n_win,
                steps_per_window=pl.steps_win, transmission=T,
                handoff='on device (3 complex components x overlap planes)',
                full_plan_windows=19,
                full_plan_seconds_extrapolated=wall / pl.n_win * 19,
                extrapolation='every window of the 19-window plan has the same size and step count as the '
                              'measured ones (the last is flush with the domain end), so the whole plan takes '
                              '19 / windows of the measured wall time at the measured rate',
                concurrent_members=conc, err_vs_reference=stitch_vs_reference())


def run_serving(count=32, seed=4):
    """The serving_stream workload: the first `count` requests of the seeded Poisson stream (mean 50
    req/s; 70 % 2D, 25 % 3D, 5 % stitch) replayed in real time through
    serve.Server (160 GB budget).  Latency = completion (result on the host)
    minus arrival."""
    import torch
    from lens_sensor_b200.serve import Request, Server, summary
    from lens_sensor_b200.workloads import serving_stream
    reqs = [Request(i, k, sp, n, t) for i, (k, sp, n, t) in enumerate(serving_stream(seed=seed, count=count))]
    srv = Server()
    done = srv.run(reqs)
    out = summary(done)
    torch.cuda.empty_cache()
    out.update(workload=f'serving_stream: first {count} requests of the seeded Poisson stream (50 req/s): '
                        f'{sum(r.kind == "2d" for r in reqs)} 2D, {sum(r.kind == "3d" for r in reqs)} 3D, '
                        f'{sum(r.kind == "stitch" for r in reqs)} stitch',
               unit=UNIT, value=out['cell_updates_per_s'], budget_bytes=srv.budget, slots3d=srv.slots3d,
               arrival_span_s=max(r.arrival for r in reqs), gpu_launches=srv.launched)
    return out


def ours_arm(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device('cuda', local))
        pg = dist
    from lens_sensor_b200.solver3d import Solve3D
    from lens_sensor_b200.workloads import waveguide3d_tm
    spec, steps_total = waveguide3d_tm()
    cells = spec.nx * spec.ny * spec.nz
    eng = args.engine3d
    solve = Solve3D(spec, steps_total, comps=(0, 1, 2), engine=eng)
    W = max(3, args.warmup)
    W += W % 2                        # spans of whole launch pairs for the two-step kernel
    ka, kb = split_steps(args.steps, steps_total, solve.n_acc)
    ka = min(ka, solve.dft[0] - W)
    kb = min(kb, solve.n_acc)
    ka -= ka % 2
    kb -= kb % 2
    K = ka + kb
    uuid = None
    try:
        uuid = 'GPU-' + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = Clocks(uuid)
    time.sleep(0.5)
    solve.run(W)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    l0 = solve.launches
    # events on the stream the kernels run on (torch's current stream): segment A is
    # ka steps before the averaging and DFT windows (one step-kernel launch each),
    # segment B the last kb steps of the schedule (window epilogue and |E|^2 passes)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    solve.n = W
    solve.run(W + ka)
    ev[1].record()
    solve.n = steps_total - kb
    solve.run(steps_total)
    ev[2].record()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ck = clocks.stop()
    launches = solve.launches - l0
    ms_a = ev[0].elapsed_time(ev[1])
    ms = max_over_ranks(ms_a + ev[1].elapsed_time(ev[2]), pg)
    value = job_rate(cells, K, ws, ms * 1e-3)
    # algorithmic bytes of the whole mix: 72 B per cell update (6 fields R+W, 3 ce + 3 D
    # read), +12 B (E re-read) +16 B per accumulated component (complex float32 R+W) on
    # window steps, +20 B per |E|^2 accumulation pass
    n_iavg = len(solve.iavg_steps(W, W + ka)) + len(solve.iavg_steps(steps_total - kb, steps_total))
    alg = cells * (72 * K + (12 + 16 * len(solve.comps)) * kb + 20 * n_iavg)
    assert not solve.iavg_steps(W, W + ka) and W + ka <= solve.prev[0]
    peak, peak_src = peaks()
    # roofline of the dominant kernel (the fused step, one launch per segment-A step)
    steps_per_launch = 2 if eng == 'tb' else 1
    t_launch = ms_a * 1e-3 / max(ka // steps_per_launch, 1)
    achieved = 72.0 * cells * steps_per_launch / t_launch / 1e9
    traffic = None
    try:
        name = 'tb3d' if eng == 'tb' else 'yee3d'
        with open(os.path.join(ROOT, 'profiles', f'{name}_waveguide3d_tm_traffic.json')) as f:
            traffic = json.load(f).get('bytes_per_launch')
    except Exception:
        pass
    # end to end through the public API: host setup, H2D, the whole 4000-step schedule, D2H of phasors
    del solve
    torch.cuda.empty_cache()
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(spec, steps_total, cells, ws, pg, engine=eng)
    planar = run_planar2d(cpu=(rank == 0 and not args.no_cpu)) if (ws == 1 and not args.no_planar) else None
    batched = run_batched(count=args.batch_instances) if (ws == 1 and not args.no_batch) else None
    stitch = run_stitch(args.stitch_windows) if (ws == 1 and not args.no_stitch) else None
    serving = run_serving(args.serve_requests) if (ws == 1 and not args.no_serve) else None
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        v, info = cpu_baseline(spec)
        cpu = dict(value=v, unit=UNIT, cores=info['cores'], kind='port', sample=info['sample'])
    if rank == 0:
        line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=ws, steps=K, warmup=W,
                    ms_per_step=ms / K, higher_is_better=True, scaling='weak', vs_baseline=None,
                    dtype='f32', data='synthetic',
                    config=dict(workload=WORKLOAD, cells=cells, steps_total=steps_total,
                                timed_steps_outside_dft=ka, timed_steps_in_dft=kb,
                                l2='inputs larger than L2: ~1.7 GB of fields and coefficients stream per step',
                                parallelism=f'replicas{ws}' if ws > 1 else 'single'),
                    roofline=dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s',
                                  frac=achieved / peak, traffic=traffic, peak_source=peak_src,
                                  kernel=('tb3d (two steps per launch, epilogues fused)' if eng == 'tb'
                                          else 'yee3d (fused step)'),
                                  steps_per_launch=steps_per_launch,
                                  alg_bytes_per_launch=72 * cells * steps_per_launch,
                                  launch_ms=t_launch * 1e3,
                                  mix_alg_bytes_per_cell_update=alg / (cells * K),
                                  mix_achieved=alg / (ms * 1e-3) / 1e9),
                    cpu_baseline=cpu, e2e=e2e, clocks=ck, gpu_launches=launches, planar2d=planar, batched=batched,
                    stitch=stitch, serving=serving)
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=1000)
    ap.add_argument('--warmup', type=int, default=20)
    ap.add_argument('--impl', default='ours', choices=('ours', 'reference'))
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline sample')
    ap.add_argument('--engine3d', default='fused', choices=('fused', 'tb'),
                    help='3D step: fused single step per launch, or two steps per launch (tb)')
    ap.add_argument('--no-e2e', action='store_true', help='skip the end-to-end solve (profiling runs)')
    ap.add_argument('--no-batch', action='store_true', help='skip the batched 2D sweep (sweep2d)')
    ap.add_argument('--no-planar', action='store_true', help='skip the 2D single-grid solve (planar2d_te)')
    ap.add_argument('--no-stitch', action='store_true', help='skip the 3D stitch (stitch3d_plan windows)')
    ap.add_argument('--batch-instances', type=int, default=256,
                    help='instances of the sweep2d sweep (fewer: a small case for profiling)')
    ap.add_argument('--stitch-windows', type=int, default=3, help='stitch windows (0: all 19 of stitch3d_plan)')
    ap.add_argument('--no-serve', action='store_true', help='skip the serving stream (serving_stream)')
    ap.add_argument('--serve-requests', type=int, default=32, help='requests of the serving stream')
    args = ap.parse_args()
    if args.impl == 'reference':
        reference_arm(args)
    else:
        ours_arm(args)


if __name__ == '__main__':
    main()
