"""Drop-in for planar_3d/fdtd3d_core.py: run_3d (full-domain CPML CW solve) and
save_results_3d, with the time loop on the B200 engine.

Same signature, physics setup (legacy tear film or free layer stack, KAPPA
absorption, sub-pixel sphere bead, staggered harmonic coefficients, CPML,
Gaussian VCSEL Huygens source), schedule (step count, detector boxes, Iavg
sampling, CW DFT over the last 8 periods with the z mid-plane convergence test
and its extension, snapshots) and the same result dictionary and output files
as the reference (fdtd3d_core.py:793-1308, 2218-2461).  Supported:
boundary='cpml', source_type='cw', no CAD, no calibration run, driven-component
snapshots (save_vector=False); other requests raise NotImplementedError.
"""
import os
import pickle
import time

import numpy as np
import torch

from . import engine as E
from .geometry import Sphere, Spec3D, Stack, build_3d
from .physics import C0, cornea_default, n_at
from .stitch3d import StitchPlan, StitchSolve

# module switches the reference's driver sets (fdtd3d_core.py:52-60)
KAPPA = {}
SRC_CORE_ONLY = False
BEAD_SUBPIXEL = True
LASER_POWER_MW = 20.0
N_G_FACTOR = 1.10
CW_TOL = 0.01
CW_MAX_EXTEND = 2.0
N_AIR = 1.0
VCSEL_NPZ_KEYS = ('laser_power_mw', 'p_src_si', 'coupling_efficiency', 'facet_reflection',
                  'vcsel_distance_um', 'vcsel_air_um', 'vcsel_waist_um', 'vcsel_waist_z_um', 'x_facet_um')


def _stack_lossy(stack):
    """KAPPA (legacy keys) or a stack layer with Im(n) > 0 (fdtd3d_core.py:61-70)."""
    if any(v > 0 for v in (KAPPA or {}).values()):
        return True
    return bool(stack) and any(complex(Ly['n']).imag > 0 for Ly in stack)


def _resolve_tear_um(tear_um, t_lip_um, t_aq_um, t_mu_um, n_cells, dx_um, cornea_um=1.5, stack=None):
    """Depth below the core: explicit, else layers + cornea margin + absorber (fdtd3d_core.py:734-754)."""
    if tear_um is not None:
        return float(tear_um)
    layers = sum(float(Ly['t_um']) for Ly in stack) if stack is not None else t_lip_um + t_aq_um + t_mu_um
    return layers + cornea_um + n_cells * dx_um


def _legacy_stack(t_lip_um, n_lip, t_aq_um, n_aq, t_mu_um, n_mu):
    """Result-dict stack of the three fixed layers (layer_stack.py:77-87), KAPPA included."""
    kp = dict(KAPPA or {})
    out = []
    for nm, t, n, mat, key in (('Lipid', t_lip_um, n_lip, 'lipid', 'lip'), ('Aqueous', t_aq_um, n_aq, 'aqueous', 'aq'),
                               ('Mucin', t_mu_um, n_mu, 'mucin', 'mu')):
        if t is None or float(t) <= 1e-9:
            continue
        nc = complex(float(np.real(n)), kp.get(key, 0.0))
        out.append(dict(name=nm, t_um=float(t), n=nc, kappa=nc.imag, mat=mat))
    return out


def _layers_tuple(stack):
    """Four-value `layers` key of a custom stack (layer_stack.py:143-149)."""
    st = list(stack or [])
    t = [st[i]['t_um'] * 1e-6 if i < len(st) else 0.0 for i in range(3)]
    n2 = complex(st[1]['n']).real if len(st) > 1 else (complex(st[0]['n']).real if st else 1.333)
    return (t[0], t[1], t[2], n2)


def _stack_npz(stack):
    st = list(stack or [])
    return dict(stack_names=np.array([L['name'] for L in st] or [''], dtype=str)[:len(st)],
                stack_t_um=np.array([L['t_um'] for L in st], dtype=np.float64),
                stack_n_re=np.array([complex(L['n']).real for L in st], dtype=np.float64),
                stack_n_im=np.array([complex(L['n']).imag for L in st], dtype=np.float64))


def _guard_in_plane(i_in, src_ix, n_max, margin=5):
    lo = int(src_ix) + int(margin)
    return int(i_in) if i_in >= lo else min(lo, int(n_max) - 2)


def run_3d(label, wg_n, t_wg_um=5.0,
           t_lip_um=0.0, t_aq_um=3.5, t_mu_um=0.5,
           n_lip=1.480, n_aq=1.336, n_mu=1.342, n_co=1.376,
           lam_nm=850.0,
           lx_um=40.0, air_um=3.0, tear_um=None, lz_um=8.0,
           dx_nm=50.0, vcsel_waist_um=3.0, vcsel_waist_z_um=3.0,
           source_type='cw', n_snapshots=8, steps_factor=2.0,
           bead=None, n_sponge=None, sponge_um=1.2, sponge_alpha=0.3,
           det_in_um=None, det_out_um=None, vol_dtype='float32',
           calibrate_steps=0, wg_width_um=None, n_clad_side=N_AIR,
           save_vector=False, check_resources=False,
           pec_faces=(), end_facet_um=0.0,
           vcsel_tilt_deg=0.0, vcsel_offset_y_um=0.0, vcsel_offset_z_um=0.0,
           input_gap_um=0.0, polarization='s', allow_large=False, boundary='cpml',
           cad=None, pulse_cycles=30.0, stack=None):
    """Full 3D FDTD solve (fdtd3d_core.py:793-1308) on the GPU engine."""
    bad = [nm for nm, v in (('source_type', source_type != 'cw'), ('calibrate_steps', bool(calibrate_steps)),
                            ('save_vector', bool(save_vector)), ('cad', cad is not None),
                            ('boundary', str(boundary or '').lower() != 'cpml'),
                            ('SRC_CORE_ONLY', bool(SRC_CORE_ONLY)), ('BEAD_SUBPIXEL', not BEAD_SUBPIXEL)) if v]
    if bad:
        raise NotImplementedError(f'lens_sensor_b200.run_3d: {", ".join(bad)}: only the full-domain CPML CW '
                                  f'path runs on the B200 engine')
    t_total = time.time()
    dx = dx_nm * 1e-9
    dx_um = dx_nm / 1000.0
    LAM = lam_nm * 1e-9
    f0 = C0 / LAM
    tear_um = _resolve_tear_um(tear_um, t_lip_um, t_aq_um, t_mu_um, 10, dx_um, stack=stack)
    ly_um = t_wg_um + air_um + tear_um
    y0_um, z0_um = -tear_um, -lz_um / 2.0
    Nx, Ny, Nz = int(round(lx_um / dx_um)), int(round(ly_um / dx_um)), int(round(lz_um / dx_um))
    lossy = _stack_lossy(stack)
    kp = dict(KAPPA or {})
    cplx = (lambda n, key: complex(float(np.real(n)), kp.get(key, 0.0)) if lossy else float(np.real(n)))
    if stack is None:
        layers = ([(t_lip_um, cplx(n_lip, 'lip'))] if t_lip_um > 1e-6 else []) + \
                 [(t_aq_um, cplx(n_aq, 'aq')), (t_mu_um, cplx(n_mu, 'mu'))]
    else:
        layers = [(float(Ly['t_um']), complex(Ly['n']) if lossy else complex(Ly['n']).real) for Ly in stack]
    st = Stack(cplx(wg_n, 'wg'), t_wg_um, layers, n_co, k_sub=kp.get('co', 0.0) if lossy else 0.0,
               force_lossy=lossy)
    beads = []
    if bead is not None and bead.get('d_um', 0) > 0:
        beads.append(Sphere(bead['x_um'], bead['d_um'], cplx(bead['n'], 'bead') if lossy else bead['n'],
                            bead.get('y_um'), bead.get('z_um', 0.0)))
    pol = 'p' if str(polarization).lower() in ('p', 'tm') else 's'
    sp = Spec3D(pol, Nx, Ny, Nz, dx_nm, st, tear_um, beads, npml=10, lam_nm=lam_nm, waist_um=vcsel_waist_um,
                waist_z_um=vcsel_waist_z_um, offset_y_um=vcsel_offset_y_um, offset_z_um=vcsel_offset_z_um,
                tilt_deg=vcsel_tilt_deg, vcsel_distance_um=float(input_gap_um or 0.0), n_sponge=n_sponge,
                sponge_um=sponge_um, end_facet_um=end_facet_um or 0.0, wg_width_um=wg_width_um,
                n_clad_side=n_clad_side, pec_faces=tuple(pec_faces or ()))
    geo = build_3d(sp)
    n_sp, src_ix, dt = sp.n_sp, sp.src_ix, sp.dt
    x_src_um = src_ix * dx_um
    x_wg_start_um = geo['x_facet_um']
    air = geo['src']['air_um']
    comp = sp.src_comp
    Nj, Nk = (Ny - 1, Nz) if pol == 'p' else (Ny, Nz - 1)
    grid = E.Grid3D(Nx, Ny, Nz, dx, dt, geo['ce'], geo['da'], geo['cpml'], geo['src'], src_comp=comp,
                    pec=(1,) * 6, fused=True)
    # detector boxes (fdtd3d_core.py:1000-1027)
    det_in_um = 0.2 * lx_um if det_in_um is None else det_in_um
    det_out_um = 0.8 * lx_um if det_out_um is None else det_out_um
    j_wg0, j_wg1 = int(round((0.0 - y0_um) / dx_um)), int(round((t_wg_um - y0_um) / dx_um))
    hw = max(2, int(round(1.0 / dx_um)))

    def xrange_at(xu):
        c = int(round(xu / dx_um))
        return max(0, c - hw), min(Nx, c + hw)
    iin0, iin1 = xrange_at(det_in_um)
    iout0, iout1 = xrange_at(det_out_um)
    ci = (iin0 + iin1) // 2
    sh = _guard_in_plane(ci, max(src_ix, int(round(x_wg_start_um / dx_um))), Nx) - ci
    iin0, iin1 = iin0 + sh, min(Nx, iin1 + sh)
    det_in_um = 0.5 * (iin0 + iin1) * dx_um
    planes = {'in': max(1, (iin0 + iin1) // 2), 'out': max(1, (iout0 + iout1) // 2),
              'src_up': src_ix - 1, 'src_dn': src_ix + 3}
    # schedule (fdtd3d_core.py:1031-1046)
    steps_total = int((24.0 / (2 * np.pi * f0) + steps_factor * lx_um * 1e-6 * N_G_FACTOR * wg_n / C0) / dt)
    steps_max = int(CW_MAX_EXTEND * steps_total)
    snap_every = max(1, steps_total // max(1, n_snapshots))
    n_avg0 = steps_total // 2
    omega = 2 * np.pi * f0
    steps_per_T = max(4, int(round((1.0 / f0) / dt)))
    n_acc = min(steps_total, 8 * steps_per_T)
    kc = Nk // 2
    m_I = max(1, steps_per_T // 8)
    prev = (max(0, steps_total - 2 * n_acc), steps_total - n_acc)
    tab = E.StepTable(0, steps_max + n_acc + 1, dt, geo['src']['omega'], omega, E.cw_envelope(f0))
    zr = (n_sp, -n_sp)     # slice(n_sp, -n_sp) of each component (fdtd3d_core.py:1139-1142)
    ep = E.Epi3D(grid, boxes=[(iin0, iin1, j_wg0, j_wg1) + zr, (iout0, iout1, j_wg0, j_wg1) + zr],
                 dft=(steps_total - n_acc, steps_total), comps=(comp,), planes=planes,
                 conv=(kc, prev), iavg=True)
    vol_dt = np.float16 if vol_dtype == 'float16' else np.float32
    os.makedirs('results', exist_ok=True)
    safe = ''.join(c if (c.isalnum() or c in '-_.') else '_' for c in str(label))
    stream_paths = []

    def mmap(shape, tag):
        p = os.path.join('results', f'_stream3d_{safe}_{tag}.npy')
        stream_paths.append(p)
        return np.lib.format.open_memmap(p, mode='w+', dtype=vol_dt, shape=shape)
    n_snaps = sum(1 for nn in range(steps_total) if (nn + 1) % snap_every == 0)
    vol_buf = mmap((n_snaps, Nx, Nj, Nk), 'ez') if n_snaps else None
    fname = 'ey' if comp == 1 else 'ez'
    snap_steps, snap_times = [], []
    ksnap, n_I = 0, 0
    cw_rel_change = float('nan')
    n_last, n_prev = n_acc, prev[1] - prev[0]
    t_start = time.time()
    n, total = 0, steps_total
    while n < total:
        # next step after which the host acts: |E|^2 sample, snapshot or the window end
        ev = total - 1
        if n >= n_avg0:
            ev = min(ev, n + (-(n - n_avg0)) % m_I)
        else:
            ev = min(ev, n_avg0)
        if ksnap < n_snaps:
            ev = min(ev, n + (-(n + 1)) % snap_every)
        grid.step(tab, n, ev - n + 1, ep)
        m, n = ev, ev + 1
        if m >= n_avg0 and (m - n_avg0) % m_I == 0:
            grid.accum_e2(ep.iavg)
            n_I += 1
        if m + 1 == total and n_prev > 0 and n_last > 0:
            cw_rel_change = ep.conv_change(n_last, n_prev)
            if cw_rel_change > CW_TOL and total + n_acc <= steps_max:
                ep.restart_dft((total, total + n_acc))
                n_prev, n_last = n_last, n_acc
                total += n_acc
        if vol_buf is not None and (m + 1) % snap_every == 0 and ksnap < n_snaps:
            vol_buf[ksnap] = grid.view(fname).cpu().numpy().astype(vol_dt)
            snap_steps.append(m + 1)
            snap_times.append(time.time() - t_start)
            ksnap += 1
    steps_total = total
    grid.check_flag()          # synchronises; raises if a pipeline wait gave up
    Iavg_np = ep.iavg[:Nx, :Nj, :Nk].cpu().numpy() / max(1, n_I)
    box = ep.box_acc.double().cpu().numpy()
    P_in, P_out = float(box[0]) * dx ** 3, float(box[1]) * dx ** 3
    Tr_I = P_out / max(P_in, 1e-30)
    S_in, S_out = ep.flux('in', n_acc), ep.flux('out', n_acc)
    p_si = S_in * dx * dx
    Tr, tr_def = Tr_I, 'intensity'
    if abs(S_in) > 0:
        Tr, tr_def = S_out / S_in, 'poynting'
    if vol_buf is not None:
        vol_buf.flush()
    va = vol_buf[:ksnap] if vol_buf is not None else None
    Ecw = ((2.0 / n_acc) * ep.phasor(comp)).cpu().numpy()
    nfr_cw = max(1, ksnap if ksnap else n_snapshots)
    cw_vol = mmap((nfr_cw, Nx, Nj, Nk), 'cwvol')
    for q in range(nfr_cw):
        tk = (q / nfr_cw) * (1.0 / f0)
        cw_vol[q] = np.real(Ecw * np.exp(1j * omega * tk)).astype(vol_dt)
    cw_vol.flush()
    if stack is not None:
        rs = ([dict(Ly) for Ly in stack], True, _layers_tuple(stack))
    else:
        rs = (_legacy_stack(t_lip_um, n_lip, t_aq_um, n_aq, t_mu_um, n_mu), False,
              (t_lip_um * 1e-6, t_aq_um * 1e-6, t_mu_um * 1e-6, n_aq))
    up, dn = ep.flux('src_up', n_acc), ep.flux('src_dn', n_acc)
    p_emit, p_refl = (dn - up) * dx * dx, -up * dx * dx
    vres = dict(laser_power_mw=LASER_POWER_MW, vcsel_distance_um=float(input_gap_um or 0.0),
                vcsel_air_um=float(air), x_facet_um=float(x_wg_start_um), vcsel_waist_um=float(vcsel_waist_um),
                vcsel_waist_z_um=float(vcsel_waist_z_um), p_src_si=p_emit)
    if p_emit and p_emit > 0:
        vres.update(coupling_efficiency=p_si / p_emit, facet_reflection=p_refl / p_emit)
    return dict(**vres, scenario=label, dim='3D', P_in=P_in, P_out=P_out, p_in_si=p_si, p_in_unit='W',
                transmission=Tr, vols_array=va, vols_ex=None, vols_ey=None, vector=False,
                _stream_paths=stream_paths, snap_steps=snap_steps, snap_times=snap_times, Iavg=Iavg_np,
                cw_vol=cw_vol, view_primary='transient', f0=f0, transmission_intensity=Tr_I,
                transmission_def=tr_def, cw_rel_change=cw_rel_change, total_time=time.time() - t_total,
                steps_total=steps_total, dt=dt, dx_nm=dx_nm, lx_um=lx_um, ly_um=ly_um, lz_um=lz_um,
                y0_um=y0_um, z0_um=z0_um, t_wg_um=t_wg_um, wg_n=wg_n, layers=rs[2], stack=rs[0],
                stack_custom=rs[1], n_lip=n_lip, n_aq=n_aq, n_mu=n_mu, n_co=n_co, lam_nm=lam_nm,
                source_type=source_type, bead=(bead if bead else {}), det_in_um=det_in_um,
                det_out_um=det_out_um, x_wg_start_um=x_wg_start_um, end_facet_um=(end_facet_um or 0.0),
                x_src_um=x_src_um, polarization=pol, cad=None, cad_region=None)


def run_3d_stitched(label, wg_n, window_w_um=20.0, slide_um=12.0,
                    t_wg_um=5.0, t_lip_um=0.0, t_aq_um=3.5, t_mu_um=0.5,
                    n_lip=1.480, n_aq=1.336, n_mu=1.342, n_co=1.376,
                    lam_nm=850.0, lx_um=40.0, air_um=3.0, tear_um=None, lz_um=8.0,
                    dx_nm=50.0, vcsel_waist_um=3.0, vcsel_waist_z_um=3.0,
                    source_type='cw', n_snapshots=8,
                    bead=None, n_sponge=None, sponge_um=1.2, sponge_alpha=0.3,
                    det_in_um=None, det_out_um=None, vol_dtype='float32',
                    wg_width_um=None, n_clad_side=N_AIR,
                    vcsel_tilt_deg=0.0, vcsel_offset_y_um=0.0, vcsel_offset_z_um=0.0,
                    input_gap_um=0.0, polarization='s', boundary='cpml', cad=None,
                    return_efull=False, stack=None):
    """3D CW solve by domain decomposition along x (fdtd3d_core.py:1311-1782).

    Windows of window_w_um slide by slide_um; each runs to steady state on the
    engine (stitch3d.StitchSolve).  Window 0 carries the VCSEL source; window
    w > 0 is driven on its first O = window - slide planes by the complex Ex,
    Ey, Ez amplitudes of the previous window's overlap (cosine taper 1 -> 0),
    which stay on the device from one window to the next.  Interior window ends
    get a CPML in an absorber extension that is neither assembled nor handed
    over.  The driven component's amplitude and <|E|^2> are assembled over the
    whole length (disk memmaps, like the reference) and written out as CW phase
    frames.  Supported: boundary='cpml', no CAD; other requests raise
    NotImplementedError."""
    bad = [nm for nm, v in (('cad', cad is not None), ('boundary', str(boundary or 'cpml').lower() != 'cpml'),
                            ('SRC_CORE_ONLY', bool(SRC_CORE_ONLY)), ('BEAD_SUBPIXEL', not BEAD_SUBPIXEL)) if v]
    if bad:
        raise NotImplementedError(f'lens_sensor_b200.run_3d_stitched: {", ".join(bad)}: only the CPML '
                                  f'stitch runs on the B200 engine')
    t_total = time.time()
    dx_um = dx_nm / 1000.0
    tear_um = _resolve_tear_um(tear_um, t_lip_um, t_aq_um, t_mu_um, 10, dx_um, stack=stack)
    ly_um = t_wg_um + air_um + tear_um
    lossy = _stack_lossy(stack)
    kp = dict(KAPPA or {})
    cplx = (lambda n, key: complex(float(np.real(n)), kp.get(key, 0.0)) if lossy else float(np.real(n)))
    if stack is None:
        layers = ([(t_lip_um, cplx(n_lip, 'lip'))] if t_lip_um > 1e-6 else []) + \
                 [(t_aq_um, cplx(n_aq, 'aq')), (t_mu_um, cplx(n_mu, 'mu'))]
    else:
        layers = [(float(Ly['t_um']), complex(Ly['n']) if lossy else complex(Ly['n']).real) for Ly in stack]
    st = Stack(cplx(wg_n, 'wg'), t_wg_um, layers, n_co, k_sub=kp.get('co', 0.0) if lossy else 0.0,
               force_lossy=lossy)
    beads = []
    if bead is not None and bead.get('d_um', 0) > 0:
        beads.append(Sphere(bead['x_um'], bead['d_um'], cplx(bead['n'], 'bead') if lossy else bead['n'],
                            bead.get('y_um'), bead.get('z_um', 0.0)))
    pl = StitchPlan(st, tear_um, lx_um, ly_um, lz_um, dx_nm, window_w_um, slide_um, wg_n, pol=polarization,
                    lam_nm=lam_nm, beads=beads, n_sponge=n_sponge, sponge_um=sponge_um, input_gap_um=input_gap_um,
                    waist_um=vcsel_waist_um, waist_z_um=vcsel_waist_z_um, tilt_deg=vcsel_tilt_deg,
                    offset_y_um=vcsel_offset_y_um, offset_z_um=vcsel_offset_z_um, wg_width_um=wg_width_um,
                    n_clad_side=n_clad_side, det_in_um=det_in_um, det_out_um=det_out_um, n_g_factor=N_G_FACTOR)
    if not pl.planes_covered():
        raise NotImplementedError('lens_sensor_b200.run_3d_stitched: a detector plane falls on a window '
                                  'start (no overlap); the intensity-based fallback is not built')
    dx, f0, omega = pl.dx, pl.f0, pl.omega
    Nx_full, Nj, Nk, n_sp = pl.Nx_full, pl.Nj, pl.Nk, pl.n_sp
    # device footprint of one window (fdtd3d_core.py:1405-1450): refuse before the run
    need = pl.window_bytes(3, lossy)
    if torch.cuda.is_available():
        free = torch.cuda.mem_get_info()[0]
        if need > 0.85 * free:
            print(f'!!! ABORT: one window (~{need / 1e9:.1f} GB) does not fit into the free device memory '
                  f'({free / 1e9:.1f} GB); choose a narrower window.')
            raise SystemExit(2)
    vcell = Nx_full * Nj * Nk
    gb_tot = (vcell * 8 + max(1, n_snapshots) * vcell * (2 if vol_dtype == 'float16' else 4) + vcell * 4) / 1e9
    try:
        import shutil
        if gb_tot > 0.95 * shutil.disk_usage(os.getcwd()).free / 1e9:
            print(f'!!! ABORT: ~{gb_tot:.1f} GB of output does not fit on the disk.')
            raise SystemExit(2)
    except SystemExit:
        raise
    except Exception:
        pass
    vol_dt = np.float16 if vol_dtype == 'float16' else np.float32
    os.makedirs('results', exist_ok=True)
    safe = ''.join(c if (c.isalnum() or c in '-_.') else '_' for c in str(label))
    stream_paths = []
    ef_path = os.path.join('results', f'_stream3d_{safe}_stitch_Efull.npy')
    Efull = np.lib.format.open_memmap(ef_path, mode='w+', dtype=np.complex64, shape=(Nx_full, Nj, Nk))
    ia_path = os.path.join('results', f'_stream3d_{safe}_stitch_Iavg.npy')
    stream_paths.append(ia_path)
    Iavg = np.lib.format.open_memmap(ia_path, mode='w+', dtype=np.float32, shape=(Nx_full, Nj, Nk))

    def sink(w, g_lo, g_hi, Ew, Ia):
        Efull[g_lo:g_hi] = Ew
        Iavg[g_lo:g_hi] = Ia
        Efull.flush()
        Iavg.flush()
    job = StitchSolve(pl, E, sink)
    while not job.done:
        job.advance(pl.steps_win)
    total_time = time.time() - t_total
    nfr = max(1, n_snapshots)
    vp = os.path.join('results', f'_stream3d_{safe}_stitch_ez.npy')
    stream_paths.append(vp)
    vol_buf = np.lib.format.open_memmap(vp, mode='w+', dtype=vol_dt, shape=(nfr, Nx_full, Nj, Nk))
    snap_times = [(k / nfr) * (1.0 / f0) for k in range(nfr)]
    snap_steps = [k + 1 for k in range(nfr)]
    cs = [float(np.cos(omega * tk)) for tk in snap_times]
    sn = [float(np.sin(omega * tk)) for tk in snap_times]
    for x0 in range(0, Nx_full, 512):
        x1 = min(x0 + 512, Nx_full)
        blk = np.asarray(Efull[x0:x1])
        for k in range(nfr):
            vol_buf[k, x0:x1] = (blk.real * cs[k] - blk.imag * sn[k]).astype(vol_dt)
    vol_buf.flush()
    Iavg.flush()
    # sensor figures from <|E|^2> on single x planes (fdtd3d_core.py:1713-1719)
    det_in_um, det_out_um = pl.det_in_um, pl.det_out_um
    iin = min(max(int(round(det_in_um / dx_um)), 0), Nx_full - 1)
    iout = min(max(int(round(det_out_um / dx_um)), 0), Nx_full - 1)
    P_in = 2.0 * float(np.sum(np.asarray(Iavg[iin, pl.j_wg0:pl.j_wg1, n_sp:-n_sp]))) * dx ** 3
    P_out = 2.0 * float(np.sum(np.asarray(Iavg[iout, pl.j_wg0:pl.j_wg1, n_sp:-n_sp]))) * dx ** 3
    Tr_I = P_out / max(P_in, 1e-30)
    Tr, tr_def = Tr_I, 'intensity'
    T = job.transmission()
    if T == T:
        Tr, tr_def = T, 'poynting'
    vc = job.vcsel()
    p_si = vc['p_in']
    Efull_ret = np.array(Efull) if return_efull else None
    try:
        Efull._mmap.close()
    except Exception:
        pass
    if os.path.exists(ef_path):
        os.remove(ef_path)
    if stack is not None:
        rs = ([dict(Ly) for Ly in stack], True, _layers_tuple(stack))
    else:
        rs = (_legacy_stack(t_lip_um, n_lip, t_aq_um, n_aq, t_mu_um, n_mu), False,
              (t_lip_um * 1e-6, t_aq_um * 1e-6, t_mu_um * 1e-6, n_aq))
    vres = dict(laser_power_mw=LASER_POWER_MW, vcsel_distance_um=pl.vd, vcsel_air_um=float(job.geo0['src']['air_um']),
                x_facet_um=float(pl.x_wg_start_um), vcsel_waist_um=float(vcsel_waist_um),
                vcsel_waist_z_um=float(vcsel_waist_z_um))
    cw_ok = source_type != 'pulse' and vc['p_emit'] is not None
    p_emit = vc['p_emit'] if cw_ok else None
    vres['p_src_si'] = p_emit
    if p_emit and p_emit > 0:
        vres.update(coupling_efficiency=(p_si / p_emit) if p_si is not None else float('nan'),
                    facet_reflection=vc['p_refl'] / p_emit)
    return dict(**vres, scenario=label, dim='3D', P_in=P_in, P_out=P_out, p_in_si=p_si, p_in_unit='W',
                transmission=Tr, vols_array=vol_buf, vols_ex=None, vols_ey=None, vector=False,
                _stream_paths=stream_paths, snap_steps=snap_steps, snap_times=snap_times, Iavg=Iavg,
                total_time=total_time, steps_total=pl.steps_win * pl.n_win, dt=pl.dt, dx_nm=dx_nm, lx_um=lx_um,
                ly_um=ly_um, lz_um=lz_um, y0_um=pl.y0_um, z0_um=pl.z0_um, t_wg_um=t_wg_um, wg_n=wg_n,
                layers=rs[2], stack=rs[0], stack_custom=rs[1], n_lip=n_lip, n_aq=n_aq, n_mu=n_mu, n_co=n_co,
                lam_nm=lam_nm, source_type=source_type, bead=(bead if bead else {}), det_in_um=det_in_um,
                det_out_um=det_out_um, x_wg_start_um=pl.x_wg_start_um, end_facet_um=0.0, x_src_um=pl.x_src_um,
                polarization=pl.pol, view_primary='cw', cw_only=True, cad=None, cad_region=None, Efull=Efull_ret,
                transmission_intensity=Tr_I, transmission_def=tr_def)


def _drop_streams(res):
    """Close and delete the temporary memmaps of a result (fdtd3d_core.py:2071-2085)."""
    for q in ('vols_array', 'vols_ex', 'vols_ey', 'cw_vol', 'Iavg'):
        m = getattr(res.get(q), '_mmap', None)
        if m is not None:
            m.close()
        res[q] = None
    for pth in res.get('_stream_paths') or []:
        if os.path.exists(pth):
            os.remove(pth)


def run_3d_stitched_pulse(label, wg_n, window_w_um=20.0, slide_um=12.0, pulse_cycles=30.0,
                          pulse_tmax_fs=None, pulse_nfreq=None, pulse_dispersion=True,
                          disp_map=None, t_eval_s=None, cad=None, stack=None, **kw):
    """Transient 3D stitch by Fourier synthesis (fdtd3d_core.py:2087-2215).

    The pulse exp(-((t - 3s)/s)^2) sin(w0 t), s = pulse_cycles / f0, is taken
    apart into frequencies w_k = w0 + k dw (|w - w0| < 5.26 / s; dw =
    2 pi / (1.6 t_max) or from pulse_nfreq); each runs a CW run_3d_stitched on
    the engine and its assembled amplitude E_k (the driven component) adds
    Re(i E_k S(w_k) e^{i w_k t_j}) dw / pi to the frame at t_j, in complex64 as
    the reference does, on the device.  disp_map {parameter: material} sets
    those indices from n(lambda_k) (a (material, offset) pair adds the offset;
    'cornea_layered' the layered cornea; 'bead' the bead's n); stack layers that
    name a material follow n(lambda_k).  Results: the frames, the CW set of the
    centre frequency (8 phases), <E^2> over the frames and the transmission
    spectrum.  No CAD."""
    from .fdtd2d_core import stack_at_lambda
    if cad is not None:
        raise NotImplementedError('lens_sensor_b200.run_3d_stitched_pulse: CAD geometry is not built')
    t_total = time.time()
    lam_nm = kw.pop('lam_nm', 850.0)
    f0 = C0 / (lam_nm * 1e-9)
    w0 = 2 * np.pi * f0
    s_p = pulse_cycles / f0
    tc = 3 * s_p
    lx = kw.get('lx_um', 40.0)
    t_max = (pulse_tmax_fs * 1e-15) if pulse_tmax_fs else tc + 3 * s_p + lx * 1e-6 * wg_n * 1.15 / C0
    half = 5.26 / s_p
    dw = 2 * half / max(int(pulse_nfreq) - 1, 1) if pulse_nfreq else 2 * np.pi / (1.6 * t_max)
    m = int(np.ceil(half / dw))
    w_k = w0 + np.arange(-m, m + 1) * dw
    w_k = w_k[w_k > 0]
    lam_k = 2 * np.pi * C0 / w_k * 1e9
    G = lambda v: np.sqrt(np.pi) * s_p * np.exp(-(v * s_p) ** 2 / 4.0) * np.exp(-1j * v * tc)
    S_k = (G(w_k - w0) - G(w_k + w0)) / (2j)
    n_snap = int(kw.pop('n_snapshots', 8))
    t_j = (np.asarray(t_eval_s, dtype=np.float64) if t_eval_s is not None
           else np.linspace(0.0, t_max, max(n_snap, 8)))
    dmap = dict(disp_map or {}) if pulse_dispersion else {}
    dev = torch.device('cuda') if torch.cuda.is_available() else torch.device('cpu')
    acc, spec_T = None, []
    r_c = E_c = None
    k_c = int(np.argmin(np.abs(w_k - w0)))
    os.makedirs('results', exist_ok=True)
    safe = ''.join(c if (c.isalnum() or c in '-_.') else '_' for c in str(label))
    for k, (wk, lk, Sk) in enumerate(zip(w_k, lam_k, S_k)):
        kwk, wg_k = dict(kw), wg_n
        for par, mat in dmap.items():
            if par == 'wg_n':
                wg_k = n_at(mat, lk)
            elif par == 'bead':
                if kwk.get('bead'):
                    kwk['bead'] = dict(kwk['bead'], n=n_at(mat, lk))
            elif mat == 'cornea_layered':
                kwk[par] = cornea_default(lk)
            elif isinstance(mat, (tuple, list)):
                kwk[par] = n_at(mat[0], lk) + float(mat[1])
            else:
                kwk[par] = n_at(mat, lk)
        stk = stack_at_lambda(stack, float(lk)) if (stack is not None and pulse_dispersion) else stack
        r = run_3d_stitched(f'{label}_f{k}', wg_k, window_w_um=window_w_um, slide_um=slide_um, lam_nm=float(lk),
                            n_snapshots=1, return_efull=True, cad=None, stack=stk, **kwk)
        Ek = r.pop('Efull')
        if acc is None:
            acc = torch.zeros((len(t_j),) + Ek.shape, dtype=torch.float32, device=dev)
        c = (torch.from_numpy(np.ascontiguousarray(Ek)).to(dev) * 1j) * complex(np.complex64(Sk * dw / np.pi))
        for j, tj in enumerate(t_j):
            acc[j] += torch.real(c * complex(np.complex64(np.exp(1j * wk * tj))))
        spec_T.append(float(r['transmission']))
        if k == k_c:
            r_c, E_c = r, Ek
        _drop_streams(r)
    fr_path = os.path.join('results', f'_stream3d_{safe}_fourier_ez.npy')
    fr = np.lib.format.open_memmap(fr_path, mode='w+', dtype=np.float32, shape=tuple(acc.shape))
    for j in range(len(t_j)):
        fr[j] = acc[j].cpu().numpy()
    fr.flush()
    # the steady set at the centre frequency and <E^2> over the frames
    nfr_cw = 8
    cw_path = os.path.join('results', f'_stream3d_{safe}_fourier_cwvol.npy')
    cw_vol = np.lib.format.open_memmap(cw_path, mode='w+', dtype=np.float32, shape=(nfr_cw,) + E_c.shape)
    for q in range(nfr_cw):
        cw_vol[q] = np.real(E_c * np.complex64(np.exp(2j * np.pi * q / nfr_cw))).astype(np.float32)
    cw_vol.flush()
    ia_path = os.path.join('results', f'_stream3d_{safe}_fourier_Iavg.npy')
    Iavg = np.lib.format.open_memmap(ia_path, mode='w+', dtype=np.float32, shape=E_c.shape)
    for x0 in range(0, E_c.shape[0], 64):
        Iavg[x0:x0 + 64] = np.mean(np.asarray(fr[:, x0:x0 + 64], dtype=np.float32) ** 2, axis=0)
    Iavg.flush()
    del acc
    res = dict(r_c)
    wgt = np.abs(S_k) ** 2
    res.update(scenario=label, vols_array=fr, vols_ex=None, vols_ey=None, vector=False,
               _stream_paths=[fr_path, cw_path, ia_path], snap_steps=[int(round(t / r_c['dt'])) for t in t_j],
               snap_times=[float(t) for t in t_j], Iavg=Iavg, cw_vol=cw_vol, view_primary='transient',
               cw_only=False, source_type='pulse', lam_nm=lam_nm, total_time=time.time() - t_total,
               transmission=float(np.sum(wgt * np.array(spec_T)) / np.sum(wgt)),
               spectrum=dict(lam_nm=lam_k, T=np.array(spec_T), weight=np.abs(S_k) / np.abs(S_k).max()),
               pulse=dict(cycles=pulse_cycles, tmax_fs=t_max * 1e15, nfreq=len(w_k),
                          dispersion=bool(pulse_dispersion)))
    if stack is not None:              # the stack at lambda0
        res.update(stack=[dict(Ly) for Ly in stack], stack_custom=True, layers=_layers_tuple(stack))
    return res


def save_results_3d(result, out_dir='results', prefix='fdtd3d', material_names=None):
    """PKL summary, z mid-plane frames NPZ and full-volume NPZ (fdtd3d_core.py:2218-2461)."""
    os.makedirs(out_dir, exist_ok=True)
    tag = result['scenario']
    if material_names is None:
        material_names = ['WG', 'Lipid', 'Aqueous', 'Mucin', 'Cornea']
    mat_idx = np.array([result['wg_n'], result['n_lip'], result['n_aq'], result['n_mu'], result['n_co']],
                       dtype=np.float64)
    stk = result.get('stack')
    if stk is None:
        lay = result.get('layers') or (0.0, 3.5e-6, 0.5e-6, result.get('n_aq', 1.336))
        stk = _legacy_stack(lay[0] * 1e6, result.get('n_lip', 1.48), lay[1] * 1e6, result.get('n_aq', 1.336),
                            lay[2] * 1e6, result.get('n_mu', 1.342))
    pos = {'lipid': 1, 'aqueous': 2, 'mucin': 3}
    if result.get('stack_custom'):
        material_names = [str(material_names[0])] + [str(Ly['name']) for Ly in stk] + [str(material_names[-1])]
        mat_idx = np.array([float(np.real(result['wg_n']))] + [complex(Ly['n']).real for Ly in stk]
                           + [float(result['n_co'])], dtype=np.float64)
    elif len(material_names) > 3:
        stk = [dict(Ly, name=str(material_names[pos[Ly['mat']]])) if Ly.get('mat') in pos else dict(Ly)
               for Ly in stk]
    result['stack'] = stk
    kw_stk = _stack_npz(stk)
    big = ('vols', 'vols_array', 'vols_ex', 'vols_ey', 'Iavg', 'cw_vol', 'cad_region')
    summary = {q: v for q, v in result.items() if q not in big}
    with open(f'{out_dir}/{prefix}_{tag}.pkl', 'wb') as f:
        pickle.dump(summary, f)
    vols = result.get('vols_array')
    if vols is None or vols.shape[0] == 0:
        return None
    steps = np.array(result.get('snap_steps', []), dtype=np.int64)
    times = np.array(result.get('snap_times', []), dtype=np.float64)
    kmid = vols.shape[3] // 2
    ez_xy = vols[:, :, :, kmid].astype(np.float32)
    x_end, y_start = result['lx_um'], result['y0_um']
    y_end = result['y0_um'] + result['ly_um']
    meta = np.array([(0.0, x_end, y_start, y_end, 0, t, s) for t, s in zip(times, steps)], dtype=np.float64)
    cw_vol = result.get('cw_vol')
    cw_only = bool(result.get('cw_only', False))      # stitch results: the frames ARE the CW phases
    kw_cw_fr, kw_cw_vol = {}, {}
    if cw_vol is not None and not cw_only:
        cw_xy = np.asarray(cw_vol[:, :, :, cw_vol.shape[3] // 2]).astype(np.float32)
        f0 = result.get('f0') or (2.99792458e8 / (result.get('lam_nm', 850.0) * 1e-9))
        ncw = cw_xy.shape[0]
        meta_cw = np.array([(0.0, x_end, y_start, y_end, 0, (q / ncw) / f0, q) for q in range(ncw)],
                           dtype=np.float64)
        kw_cw_fr = dict(Ez_cw=cw_xy, meta_cw=meta_cw)
        kw_cw_vol = dict(Ez_cw=cw_vol)
    flags = dict(has_transient=np.array([0 if cw_only else 1]),
                 has_cw=np.array([1 if (cw_only or cw_vol is not None) else 0]),
                 cw_only=np.array([1 if cw_only else 0]),
                 view_primary=np.array([str(result.get('view_primary', 'transient'))]))
    spec = result.get('spectrum')
    if spec:                           # Fourier stitch: the spectrum in both NPZ (fdtd3d_core.py:2301-2308)
        pu = result.get('pulse') or {}
        flags.update(spec_lam_nm=np.asarray(spec['lam_nm'], dtype=np.float64),
                     spec_T=np.asarray(spec['T'], dtype=np.float64),
                     spec_weight=np.asarray(spec['weight'], dtype=np.float64),
                     pulse_cycles=np.array([pu.get('cycles', 0.0)]),
                     pulse_dispersion=np.array([int(bool(pu.get('dispersion', True)))]))
    bead = result.get('bead') or {}
    bd = bead.get('d_um', 0.0)
    bead_yc, bead_zc = bead.get('y_um', -bd / 2.0), bead.get('z_um', 0.0)
    kw_ia = {}
    ia = np.asarray(result.get('Iavg'))
    if ia.ndim == 3:
        kw_ia = dict(Iavg=ia[:, :, ia.shape[2] // 2].astype(np.float32), iavg_full=np.array([1]))
    kw_p = ({'p_in_si': np.array([float(result['p_in_si'])]), 'p_in_unit': np.array([str(result.get('p_in_unit', 'W'))])}
            if result.get('p_in_si') is not None else {})
    for q in VCSEL_NPZ_KEYS:
        v = result.get(q)
        try:
            if v is not None and np.isfinite(float(v)):
                kw_p[q] = np.array([float(v)])
        except (TypeError, ValueError):
            pass
    kw_ia.update(kw_p)
    common = dict(bead_x_um=np.array([bead.get('x_um', 0.0)]), bead_diameter_um=np.array([bead.get('d_um', 0.0)]),
                  bead_y_um=np.array([bead_yc]), bead_z_um=np.array([bead_zc]),
                  bead_n=np.array([bead.get('n', 0.0)]),
                  x_wg_start_um=np.array([result.get('x_wg_start_um', 0.0) or 0.0]),
                  end_facet_um=np.array([result.get('end_facet_um', 0.0) or 0.0]))
    fr_path = f'{out_dir}/{prefix}_{tag}_frames.npz'
    np.savez_compressed(fr_path, Ez=ez_xy, meta=meta, scenario=tag, **kw_ia,
                        layers=np.array(result['layers'], dtype=np.float64),
                        material_names=np.array(material_names), material_indices=mat_idx, **common,
                        x_src_um=np.array([result.get('x_src_um', 0.0) or 0.0]),
                        lam_nm=np.array([result.get('lam_nm', 850.0)]),
                        polarization=np.array([str(result.get('polarization', 's'))]),
                        **kw_stk, **kw_cw_fr, **flags)
    iavg = result['Iavg']
    iavg = iavg if getattr(iavg, 'dtype', None) == np.float32 else np.asarray(iavg).astype(np.float32)
    vol_path = f'{out_dir}/{prefix}_{tag}_vol3d.npz'
    np.savez_compressed(vol_path, **kw_p, Ez=vols, Iavg=iavg, iavg_full=np.array([1]), steps=steps, times=times,
                        dx_um=result['dx_nm'] / 1000.0, x0_um=0.0, y0_um=result['y0_um'], z0_um=result['z0_um'],
                        scenario=tag, dt=result['dt'], layers=np.array(result['layers'], dtype=np.float64),
                        material_names=np.array(material_names), material_indices=mat_idx,
                        t_wg_um=np.array([result.get('t_wg_um', 0.0)]),
                        wg_width_um=np.array([(result.get('bead') or {}).get('wg_width_um',
                                                                          result.get('wg_width_um', 0.0)) or 0.0]),
                        **common, lx_um=np.array([result.get('lx_um', 0.0)]),
                        x_src_um=np.array([result.get('x_src_um', 0.0) or 0.0]),
                        lam_nm=np.array([result.get('lam_nm', 850.0)]),
                        polarization=np.array([str(result.get('polarization', 's'))]),
                        **kw_stk, **kw_cw_vol, **flags)
    # the temporary stream memmaps go once the NPZ files are written
    for q in ('vols_array', 'vols_ex', 'vols_ey', 'cw_vol', 'Iavg'):
        a = result.get(q)
        m = getattr(a, '_mmap', None) or getattr(getattr(a, 'base', None), '_mmap', None)
        if m is not None:
            m.close()
    result['vols_array'] = result['vols_ex'] = result['vols_ey'] = None
    result['Iavg'] = None
    for p in result.get('_stream_paths') or []:
        if os.path.exists(p):
            os.remove(p)
    return fr_path, vol_path
