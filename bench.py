"""Benchmark of the direct-SCF J/K engine on one B200 (N GPUs: replicas).

Workload (one step): a complete RHF solve of (H2O)_64 in the cc-pVTZ-shaped
synthetic basis (3712 AO, s-f shells) from a SAD guess to |Delta E| <= 1e-8 Eh,
direct SCF with incremental Fock builds, Schwarz threshold 1e-13, in the fast
form (FP32 band and early screen on the builds before one full FP64 rebuild).
``value`` is SCF wall seconds per solve (CUDA events, set-up included);
``plain_fp64`` is the plain FP64 form on the same GPU; ``e2e`` repeats the
fast solve through the drop-in host API (a host SCF loop calling get_jk with
numpy arrays every cycle, the way cuobc's RHF runs under pyscf).  The
roofline object describes the dominant J/K class pair and the whole build of
one full J+K build with the converged density; the FLOP count of the plain
solve is counted on the device in the same run.  ``cpu_baseline`` is the CPU
oracle (an OpenMP C restatement of the reference's algorithm) timed on a
complete SCF of (H2O)_4 in the cc-pVDZ shape on the host cores.

--impl reference: the same SCF along the reference's own path -- its J/K
kernels (oracle/_ref: cuobc/lib/gint and gvhf compiled for sm_100a), its host
logic (oracle/ref_gpu.py, oracle/ref_scf.py: Schwarz pair lists, class-level
density screen, log-q bins, one GINTbuild_jk per class pair) and a pyscf-style
host SCF loop -- on the same GPU.  One step of this arm is one SCF cycle;
``value`` is the measured wall time of the complete SCF (set-up included)
that the timed steps contain.  Nothing of the engine library is loaded.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'SCF wall s to |ΔE|≤1e-8 Eh: mixed+batched+guess vs plain FP64, same B200'


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=1)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    p.add_argument('--nwater', type=int, default=64)
    p.add_argument('--basis', default='cc-pvtz')
    p.add_argument('--conv', type=float, default=1e-8)
    p.add_argument('--no-extras', action='store_true', help='skip e2e/roofline/cpu legs')
    p.add_argument('--per-class', action='store_true',
                   help='time one J/K build class by class (this engine, or with --impl '
                        'reference the reference kernels) and print the per-class sums')
    p.add_argument('--noscreen', action='store_true',
                   help='with --per-class: every quartet of the pair lists, no screening')
    p.add_argument('--only', default=None,
                   help='with --per-class: only the class pairs of shape li,lj,lk,ll')
    p.add_argument('--reps', type=int, default=2, help='with --per-class: builds timed')
    return p.parse_args()


def workload(args):
    from byteqc_b200.gto.mole import Mole
    from byteqc_b200.gto.basis import synthetic_basis
    from byteqc_b200.gto.geom import water_cluster
    atoms = water_cluster(args.nwater, seed=0)
    mol = Mole(atoms, synthetic_basis(args.basis, ['O', 'H']))
    mol.basis_name = args.basis.lower()
    return mol


def config(args, mol):
    return {'workload': '(H2O)%d/%s-shaped synthetic basis, plain FP64 RHF, SAD guess, DIIS, '
                        'incremental Fock' % (args.nwater, args.basis),
            'nao': mol.nao, 'natm': mol.natm, 'basis': args.basis + ' (synthetic, same shell shapes)',
            'conv_tol': args.conv, 'schwarz_cutoff': 1e-13, 'geometry_seed': 0,
            'parallelism': 'replicas' if args.gpus > 1 else 'single GPU',
            'l2': 'inputs larger than L2 (J/K matrices %.0f MB each)' % (mol.nao_nr(True) ** 2 * 8 / 1e6)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
             'clocks_event_reasons.sw_power_cap')
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + q,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm = [float(r[0]) for r in self.rows if len(r) >= 7 and r[0].replace('.', '').isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 7 and r[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for r in self.rows if len(r) >= 7
                          for i in range(4) if 'Active' in r[3 + i] and 'Not' not in r[3 + i]})
        return {'sm_mhz': float(np.median(sm)) if sm else None,
                'sm_max_mhz': max(mx) if mx else None, 'reasons': reasons,
                'samples': len(self.rows)}


FP32_BELOW = 1e-4   # bound below which the fast form evaluates quartets in FP32
EARLY_TOL = 1e-10   # screening threshold of the fast form before its final FP64 rebuild


def scf_once(mol, conv, host_loop=False, fast=False):
    """One SCF solve.  fast: the fast form (FP32 band below FP32_BELOW on the
    incremental builds, final FP64 rebuilds; learned guess when the basis has
    a trained model, i.e. the cc-pVDZ shape)."""
    import torch
    from byteqc_b200.scf import hf, guess
    guess._SAD_CACHE.clear()
    mf = hf.RHF(mol)
    mf.conv_tol = conv
    if fast:
        mf.fp32_threshold = FP32_BELOW
        mf.early_tol = EARLY_TOL
        if has_learned_guess(mol):
            mf.init_guess = 'mlp'
    if host_loop:
        e = mf.kernel_hostloop()
    else:
        e = mf.kernel()
    torch.cuda.synchronize()
    return mf, e


def has_learned_guess(mol):
    from byteqc_b200.learned.infer import weights_for
    return weights_for(mol) is not None


def roofline(mf, peak):
    """Time one full J+K build class pair by class pair with CUDA events on
    the launching stream; report the dominant class pair."""
    import ctypes
    import torch
    from byteqc_b200 import lib as L, flops
    from byteqc_b200.scf.hf import _ptr, _stream
    lib = L.load_library()
    opt = mf.opt
    C = opt.coeff_dev
    dmc = (C @ mf.dm @ C.T)[None].contiguous()
    nao = dmc.shape[-1]
    dm_cond = torch.empty((opt.mol.nbas, opt.mol.nbas), dtype=torch.float64, device=dmc.device)
    lib.BQCdm_cond(_ptr(dmc), 1, nao, _ptr(opt._mem['ao_loc']), opt.mol.nbas, _ptr(dm_cond), _stream())
    dm_max = float(dm_cond.max())
    vj = torch.zeros_like(dmc)
    vk = torch.zeros_like(dmc)
    qh = opt.pair_q_host.ctypes.data_as(ctypes.c_void_p)
    bp = ctypes.cast(opt.bpcache, ctypes.c_void_p)
    cnt = torch.zeros(1, dtype=torch.int64, device=dmc.device)
    rows = []
    total_t = total_f = 0.
    for cij in range(opt.ncptype):
        for ckl in range(cij + 1):
            if opt.cptype[cij][3] == 0 or opt.cptype[ckl][3] == 0:
                continue
            cnt.zero_()
            lib.BQCcount_quartets(bp, cij, ckl, _ptr(opt.pair_q), qh, _ptr(dm_cond), dm_max,
                                  opt.direct_scf_tol, _ptr(cnt), _stream())
            nq = int(cnt.item())
            if nq == 0:
                continue
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record()
            err = lib.BQCbuild_jk_class(bp, cij, ckl, _ptr(opt.pair_q), qh, _ptr(dm_cond), dm_max,
                                        _ptr(vj), _ptr(vk), _ptr(dmc), nao, 1,
                                        opt.direct_scf_tol, 0., None, _stream())
            ev1.record()
            torch.cuda.synchronize()
            assert err == 0
            ms = ev0.elapsed_time(ev1)
            li, lj, np_ij, _ = opt.cptype[cij]
            lk, ll, np_kl, _ = opt.cptype[ckl]
            f = nq * flops.quartet_flops(li, lj, lk, ll, np_ij, np_kl)
            rows.append({'class': '(%s%s|%s%s)' % tuple('spdf'[x] for x in (li, lj, lk, ll)),
                         'nprim': [np_ij, np_kl], 'quartets': nq, 'ms': ms, 'flops': f,
                         'prim_quartets': nq * np_ij * np_kl})
            total_t += ms
            total_f += f
    rows.sort(key=lambda r: -r['ms'])
    top = rows[0]
    achieved = top['flops'] / (top['ms'] * 1e-3) / 1e12
    return {
        'bound': 'fp64', 'unit': 'TFLOP/s', 'achieved': round(achieved, 3),
        'peak': round(peak / 1e12, 3), 'frac': round(achieved * 1e12 / peak, 4),
        'traffic': TRAFFIC.get(top['class']),
        'kernel': 'J/K class pair %s nprim %s (%.1f%% of the build)' % (
            top['class'], top['nprim'], 100 * top['ms'] / total_t),
        'peak_source': 'measured DFMA microbenchmark (BQCfp64_fma_peak) on this GPU',
        'build': {'ms': round(total_t, 2), 'tflops': round(total_f / (total_t * 1e-3) / 1e12, 3),
                  'frac': round(total_f / (total_t * 1e-3) / peak, 4),
                  'quartets': int(sum(r['quartets'] for r in rows)),
                  'quartets_per_s': float('%.4g' % (sum(r['quartets'] for r in rows) / (total_t * 1e-3))),
                  'prim_quartets_per_s': float('%.4g' % (sum(r['prim_quartets'] for r in rows)
                                                         / (total_t * 1e-3)))},
        'top_classes': [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in r.items()}
                        for r in rows[:6]],
    }


def jk_flops(opt, dm_ao):
    """Algorithmic FLOPs of one J/K build of opt for the AO density dm_ao
    (surviving quartets counted on the device per class pair)."""
    import ctypes
    import torch
    from byteqc_b200 import lib as L, flops
    from byteqc_b200.scf.hf import _ptr, _stream
    lib = L.load_library()
    C = opt.coeff_dev
    dmc = (C @ dm_ao @ C.T)[None].contiguous()
    nao = dmc.shape[-1]
    dm_cond = torch.empty((opt.mol.nbas, opt.mol.nbas), dtype=torch.float64, device=dmc.device)
    lib.BQCdm_cond(_ptr(dmc), 1, nao, _ptr(opt._mem['ao_loc']), opt.mol.nbas, _ptr(dm_cond), _stream())
    dm_max = float(dm_cond.max())
    qh = opt.pair_q_host.ctypes.data_as(ctypes.c_void_p)
    bp = ctypes.cast(opt.bpcache, ctypes.c_void_p)
    cnt = torch.zeros(1, dtype=torch.int64, device=dmc.device)
    tot = 0.
    for cij in range(opt.ncptype):
        for ckl in range(cij + 1):
            if opt.cptype[cij][3] == 0 or opt.cptype[ckl][3] == 0:
                continue
            cnt.zero_()
            lib.BQCcount_quartets(bp, cij, ckl, _ptr(opt.pair_q), qh, _ptr(dm_cond), dm_max,
                                  opt.direct_scf_tol, _ptr(cnt), _stream())
            nq = int(cnt.item())
            if nq:
                li, lj, np_ij, _ = opt.cptype[cij]
                lk, ll, np_kl, _ = opt.cptype[ckl]
                tot += nq * flops.quartet_flops(li, lj, lk, ll, np_ij, np_kl)
    return tot


def cpu_oracle_scf(threads):
    """The CPU oracle on a bounded sample: a complete RHF of (H2O)_4 in the
    cc-pVDZ shape (96 AO) to |Delta E| < 1e-8 with exact J/K (no screening)
    on `threads` host threads.  Returns (seconds, energy, cycles, sample)."""
    from byteqc_b200.gto.mole import Mole
    from byteqc_b200.gto.basis import synthetic_basis
    from byteqc_b200.gto.geom import water_cluster
    from oracle import oracle
    mol = Mole(water_cluster(4, seed=0), synthetic_basis('cc-pvdz', ['O', 'H']))
    t0 = time.perf_counter()
    e, _, cycles = oracle.rhf(mol, conv_tol=1e-8, nthreads=threads)
    t = time.perf_counter() - t0
    return t, e, cycles, ('(H2O)4/cc-pvdz-shaped (96 AO, seed 0): one complete RHF to |dE| < 1e-8 '
                          'from the core guess, exact J/K every cycle, %d threads; %d cycles' % (
                              threads, cycles))


# DRAM bytes per launch of the J/K kernels (dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu --set full capture of one launch of the
# class at (H2O)_64 / cc-pVTZ shape on the jk.py density), by class
TRAFFIC = {'(ps|ss)': 72824320 + 38084352, '(dp|ps)': 300668672 + 132837376,
           '(fp|dp)': 570294016 + 3547033000}


def main():
    args = parse()
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))

    if args.per_class:
        if rank == 0:
            per_class(args)
        return
    if args.impl == 'reference':
        if rank == 0:
            run_reference(args)
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=__import__('datetime').timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    from byteqc_b200 import lib as L
    lib = L.load_library()
    mol = workload(args)

    for _ in range(args.warmup):
        scf_once(mol, args.conv, fast=True)

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = lib.BQClaunch_counter()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record()
            mf, e = scf_once(mol, args.conv, fast=True)
            ev1.record()
            torch.cuda.synchronize()
            times.append(ev0.elapsed_time(ev1) / 1e3)
    launches = lib.BQClaunch_counter() - launches0
    t_step = float(np.mean(times))
    if world > 1:
        t_step = max_over_ranks(t_step, 'cuda')
        torch.distributed.barrier()

    line = {'metric': METRIC, 'value': round(t_step, 3), 'unit': 's', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': round(t_step * 1e3, 1),
            'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic',
            'form': 'fast: incremental builds with FP32 for quartets with bound < %g and '
                    'screening at %g, then one full FP64 rebuild and FP64 incremental builds at '
                    '1e-13 to convergence%s' % (
                        FP32_BELOW, EARLY_TOL, '; learned initial density (SAD fallback)'
                        if has_learned_guess(mol) else
                        '; SAD guess (no learned model for this basis shape)'),
            'config': config(args, mol), 'clocks': clk.summary(), 'gpu_launches': int(launches),
            'scf': {'energy': e, 'cycles': mf.cycles, 'converged': bool(mf.converged),
                    'jk_s': round(mf.timings.get('jk', 0), 3)}}

    if not args.no_extras and rank == 0:
        extras(args, mol, mf, e, t_step, line, lib)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def extras(args, mol, mf, e, t_step, line, lib):
    """The legs beside the timed steps (rank 0): plain FP64 form, e2e through
    the host API, roofline, J/K build on the reference's timing density with
    the cross-check against the reference arm's output, FLOPs of the plain
    solve counted on the device, and the CPU oracle baseline."""
    import torch
    # the plain FP64 form on the same GPU, same workload; its J/K input
    # densities are kept for the FLOP count
    from byteqc_b200.scf import hf, guess
    guess._SAD_CACHE.clear()
    mf_p = hf.RHF(mol)
    mf_p.conv_tol = args.conv
    dens = []
    mf_p.jk_hook = lambda d, fp32_below: dens.append(d.clone())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    e_p = mf_p.kernel()
    ev1.record()
    torch.cuda.synchronize()
    t_plain = ev0.elapsed_time(ev1) / 1e3
    line['plain_fp64'] = {'value': round(t_plain, 3), 'unit': 's', 'cycles': mf_p.cycles,
                          'energy': e_p, 'jk_s': round(mf_p.timings.get('jk', 0), 3),
                          'speedup_fast_vs_plain': round(t_plain / t_step, 3),
                          'energy_diff_fast_vs_plain': abs(e - e_p)}
    # e2e through the drop-in host API
    t0 = time.perf_counter()
    mf_h, e_h = scf_once(mol, args.conv, host_loop=True, fast=True)
    t_e2e = time.perf_counter() - t0
    h2d, d2h = mf_h.host_bytes
    line['e2e'] = {'value': round(t_e2e, 3), 'unit': 's', 'h2d_bytes_per_step': int(h2d),
                   'd2h_bytes_per_step': int(d2h),
                   'path': 'host SCF loop calling get_jk(mol, dm_host) every cycle',
                   'energy_diff_vs_device_loop': abs(e_h - e)}
    peak = ctypes_peak(lib)
    line['roofline'] = roofline(mf, peak)
    # FLOPs of the plain solve's J/K builds, counted on its own densities
    f_scf = sum(jk_flops(mf_p.opt, d) for d in dens)
    del dens
    line['scf']['plain_jk_flops'] = f_scf
    line['scf']['plain_jk_builds'] = mf_p.cycles
    line['scf']['plain_jk_tflops'] = round(f_scf / max(mf_p.timings.get('jk', 1e-9), 1e-9) / 1e12, 3)
    line['scf']['plain_jk_frac_of_fp64_peak'] = round(
        f_scf / max(mf_p.timings.get('jk', 1e-9), 1e-9) / peak, 4)
    # one J/K build on the density of the reference's timing script; the
    # reference arm (run first by the driver) leaves its J/K and SCF energy
    opt = mf.opt
    dmc = jkpy_density(opt)
    line['jk_build'] = {'s': round(time_build(lambda: opt.jk_cart(dmc)), 3),
                        'density': JKPY_DENSITY, 'tol': opt.direct_scf_tol}
    line['jk_build']['reference_check'] = reference_check(args, opt, dmc, e_p)
    # the batched form on its own configuration: 256 seeded (H2O)_k, k in
    # [1, 12], cc-pVDZ shape, in one batched solve, against one-by-one solves
    line['batched'] = batched_leg()
    # CPU baseline: the oracle on a bounded sample, host cores
    threads = os.cpu_count() or 1
    t_cpu, e_cpu, cyc, desc = cpu_oracle_scf(threads)
    line['cpu_baseline'] = {'value': round(t_cpu, 2), 'unit': 's', 'cores': threads,
                            'kind': 'port', 'sample': desc}
    # the same sample on this engine, for a like-for-like ratio
    from byteqc_b200.gto.mole import Mole
    from byteqc_b200.gto.basis import synthetic_basis
    from byteqc_b200.gto.geom import water_cluster
    small = Mole(water_cluster(4, seed=0), synthetic_basis('cc-pvdz', ['O', 'H']))

    def small_scf():
        m = hf.RHF(small)
        m.conv_tol = 1e-8
        m.init_guess = '1e'
        return m.kernel()
    small_scf()
    ev0.record()
    e_s = small_scf()
    ev1.record()
    torch.cuda.synchronize()
    line['cpu_baseline']['same_sample_on_gpu_s'] = round(ev0.elapsed_time(ev1) / 1e3, 3)
    line['cpu_baseline']['energy_diff_gpu_vs_oracle'] = abs(e_s - e_cpu)


def batched_leg(nmol=256, nseq=64, conv=1e-8):
    """Molecules/s of one batched solve of nmol seeded (H2O)_k (k uniform in
    [1, 12], cc-pVDZ shape) against one-by-one plain solves of the first nseq
    of them, and the largest energy difference between the two."""
    import torch
    from byteqc_b200.scf import batched, hf, guess
    mols = batched.batch_systems(nmol)
    batched.BatchedRHF(mols[:2]).kernel()     # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mf = batched.BatchedRHF(mols)
    mf.conv_tol = conv
    e = mf.kernel()
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    es = []
    t0 = time.perf_counter()
    for m in mols[:nseq]:
        one = hf.RHF(m)
        one.conv_tol = conv
        es.append(one.kernel())
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    return {'config': '%d x (H2O)_k, k uniform in [1, 12], cc-pvdz-shaped (%d AO in total)' % (
                nmol, sum(m.nao for m in mols)),
            'batched_s': round(t_batch, 3), 'molecules_per_s': round(nmol / t_batch, 2),
            'cycles': mf.cycles, 'converged': bool(mf.converged),
            'sequential_molecules_per_s': round(nseq / t_seq, 2), 'sequential_timed': nseq,
            'speedup': round((nmol / t_batch) / (nseq / t_seq), 3),
            'max_energy_diff': float(np.max(np.abs(np.asarray(es) - np.asarray(e)[:nseq])))}


REF_OUT = os.path.join(os.environ.get('TMPDIR', '/tmp'), 'byteqc_b200_reference_%s.npz')


def _ref_key(args):
    return '%dw_%s' % (args.nwater, args.basis.replace('*', 's'))


def reference_check(args, opt, dmc, e_plain):
    """J/K of the timing density and the SCF energy against what the
    reference arm computed on the same workload (its file, when present):
    max |dJ|, max |dK| in the AO basis and |dE|.  The two builds screen
    differently (per quartet here, per class pair and log-q bin there), so
    they differ by at most what either screen drops."""
    path = REF_OUT % _ref_key(args)
    if not os.path.exists(path):
        return {'skipped': 'the reference arm has not run on this box'}
    import torch
    ref = np.load(path)
    J, K = opt.jk_cart(dmc)
    C = opt.coeff_dev
    J = (C.T @ J[0] @ C).cpu().numpy()
    K = (C.T @ K[0] @ C).cpu().numpy()
    dj = float(abs(J - ref['J']).max())
    dk = float(abs(K - ref['K']).max())
    out = {'max_abs_dJ': dj, 'max_abs_dK': dk, 'max_abs_J': float(abs(ref['J']).max()),
           'bound': SCREEN_BOUND, 'within_bound': dj < SCREEN_BOUND and dk < SCREEN_BOUND}
    if 'energy' in ref.files:
        out['scf_energy_diff_vs_reference'] = abs(float(ref['energy']) - e_plain)
    return out


# Bound on the difference of two J/K builds that both drop only quartets
# whose estimate q_ij q_kl max|D| is below 1e-13: a J or K element collects at
# most ~1e4 such dropped contributions at this size.
SCREEN_BOUND = 1e-8


def run_reference(args):
    """The reference arm: the reference's SCF path with its own GPU kernels
    (see the module doc).  Steps are SCF cycles: W untimed cycles of the
    workload's SCF, then a fresh SCF (set-up included) timed to convergence,
    followed by repeats of its last cycle until K steps are done."""
    import torch
    from oracle import ref_gpu
    base = {'impl': 'reference', 'metric': METRIC}
    if not torch.cuda.is_available():
        print(json.dumps(dict(base, unavailable='no CUDA device')))
        return
    if not ref_gpu.available():
        print(json.dumps(dict(base, unavailable='oracle/_ref not built: the reference sources '
                                                'were absent when the package was built')))
        return
    from oracle.ref_scf import RefSCF
    torch.cuda.set_device(0)
    mol = workload(args)
    threads = os.cpu_count() or 1
    if args.warmup > 0:
        warm = RefSCF(mol, conv_tol=args.conv, max_cycle=args.warmup)
        warm.kernel()
        warm.close()
    torch.cuda.synchronize()
    steps = 0
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        ref = RefSCF(mol, conv_tol=args.conv)
        e = ref.kernel()
        torch.cuda.synchronize()
        t_scf = time.perf_counter() - t0
        steps = ref.cycles
        while steps < args.steps:
            ref.repeat_cycle()
            steps += 1
        torch.cuda.synchronize()
        t_all = time.perf_counter() - t0
    nao0 = mol.nao
    nao_c = ref.opt.coeff.shape[0]
    # host <-> device bytes of one cycle along the reference path: D in, D' back
    # for the class screen, J and K back; F and S in and C, e back for eig
    h2d = 8 * (nao0 * nao0 + 2 * nao0 * nao0)
    d2h = 8 * (nao_c * nao_c + 2 * nao0 * nao0 + nao0 * nao0 + nao0)
    line = dict(base, **{
        'value': round(t_scf, 3), 'unit': 's', 'n_gpus': args.gpus, 'steps': steps,
        'warmup': args.warmup, 'ms_per_step': round(t_all / steps * 1e3, 1),
        'higher_is_better': False, 'dtype': 'f64', 'data': 'synthetic',
        'config': config(args, mol), 'clocks': clk.summary(),
        'step': 'one SCF cycle of the reference path; value = wall seconds of the complete '
                'SCF (set-up, Schwarz pair lists, guess, %d cycles to |dE| < %g) inside the '
                'timed steps' % (ref.cycles, args.conv),
        'cpu_baseline': {'value': round(t_scf, 3), 'unit': 's', 'cores': threads,
                         'kind': 'reference',
                         'sample': 'the complete workload SCF: the reference J/K kernels '
                                   '(oracle/_ref) on the GPU, host SCF loop on %d host '
                                   'threads' % threads},
        'e2e': {'value': round(t_scf, 3), 'unit': 's', 'h2d_bytes_per_step': h2d,
                'd2h_bytes_per_step': d2h},
        'scf': {'energy': e, 'cycles': ref.cycles, 'converged': bool(ref.converged),
                'setup_s': round(ref.timings.get('setup', 0.), 3),
                'pair_lists_s': round(ref.timings.get('vhfopt', 0.), 3),
                'cycle_s': [round(x, 3) for x in ref.cycle_s]}})
    # one J/K build on the density of the reference's timing script
    # (cuobc/test/jk.py), timed; J, K and the SCF energy are left for the
    # engine arm's cross-check
    try:
        rng = np.random.default_rng(2341)
        dm = rng.random((nao0, nao0))
        dm = 0.1 * (dm + dm.T)
        C = ref.coeff
        dmc = (C @ torch.as_tensor(dm, device='cuda') @ C.T)[None].contiguous()
        tasks = ref.jk.tasks(dmc)
        out = {}
        t = time_build(lambda: out.setdefault('jk', ref.jk.jk_cart(dmc, tasks=tasks)), reps=1)
        J, K = ref.jk.jk_cart(dmc, tasks=tasks)
        np.savez(REF_OUT % _ref_key(args), J=(C.T @ J[0] @ C).cpu().numpy(),
                 K=(C.T @ K[0] @ C).cpu().numpy(), energy=e)
        line['reference_gpu'] = {
            'jk_build_s': round(t, 3), 'density': JKPY_DENSITY, 'launches': len(tasks),
            'what': 'GINTbuild_jk of the reference (cuobc/lib/gvhf, cuobc/lib/gint) built for '
                    'sm_100a, driven by the restated host logic of cuobc/scf/hf.py get_jk '
                    '(log-q bins, class-level density screen); same B200, CUDA events'}
    except Exception as exc:   # report, never fail the line
        line['reference_gpu'] = {'unavailable': '%s: %s' % (type(exc).__name__, exc)}
    ref.close()
    print(json.dumps(line))


def per_class(args):
    """One J/K build of the workload on the jk.py density, class pair by class
    pair (CUDA events on the launching stream), summed per class shape
    li lj lk ll; the last of --reps builds is printed.  With --impl reference
    the reference's kernels run over the pair lists of its own host logic
    (oracle/ref_gpu.py), without the engine library; with --noscreen both
    evaluate every quartet of their lists (no density screen, one bin)."""
    import ctypes
    import torch
    torch.cuda.set_device(0)
    mol = workload(args)
    only = tuple(int(x) for x in args.only.split(',')) if args.only else None
    rng = np.random.default_rng(2341)
    dm = rng.random((mol.nao, mol.nao))
    dm = torch.as_tensor(0.1 * (dm + dm.T), device='cuda')
    res, tot = {}, 0.
    if args.impl == 'reference':
        from oracle import ref_gpu
        opt = ref_gpu.RefVHFOpt(mol).build()
        ref = ref_gpu.RefJK(opt)
        C = torch.as_tensor(opt.coeff, device='cuda')
        dmc = (C @ dm @ C.T)[None].contiguous()
        tasks = ref.tasks(dmc)
        nbins = ref.nbins
        if args.noscreen:
            nb = ref.pairs_locs[1:] - ref.pairs_locs[:-1]
            tasks = [(i, j, np.array([0, nb[i]], np.int32), np.array([0, nb[j]], np.int32))
                     for i in range(opt.ncptype) for j in range(i + 1) if nb[i] and nb[j]]
            nbins = 1
        lt = [(int(opt.uniq_l_ctr[p, 0]), int(opt.uniq_l_ctr[q, 0]))
              for p in range(len(opt.uniq_l_ctr)) for q in range(p + 1)]
        vj = torch.zeros_like(dmc)
        vk = torch.zeros_like(dmc)
        vp = lambda x: x.ctypes.data_as(ctypes.c_void_p)
        tp = lambda t: ctypes.c_void_p(t.data_ptr())
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        jobs = []
        for cij, ckl, bi, bk in tasks:
            shape = lt[cij] + lt[ckl]
            if only is None or shape in (only, only[2:] + only[:2]):
                jobs.append((shape, lambda cij=cij, ckl=ckl, bi=bi, bk=bk: ref.lv.GINTbuild_jk(
                    ref.bp_gpu, tp(vj), tp(vk), tp(dmc), ctypes.c_int(dmc.shape[-1]), ctypes.c_int(1),
                    vp(bi), vp(bk), ctypes.c_int(nbins), ctypes.c_int(cij), ctypes.c_int(ckl), stream)))
    else:
        from byteqc_b200 import lib as L
        from byteqc_b200.scf import hf
        from byteqc_b200.scf.hf import _ptr, _stream
        lib = L.load_library()
        opt = hf._VHFOpt(mol).build()
        C = opt.coeff_dev
        dmc = (C @ dm @ C.T)[None].contiguous()
        nao = dmc.shape[-1]
        dm_cond = torch.empty((opt.mol.nbas, opt.mol.nbas), dtype=torch.float64, device='cuda')
        lib.BQCdm_cond(_ptr(dmc), 1, nao, _ptr(opt._mem['ao_loc']), opt.mol.nbas, _ptr(dm_cond),
                       _stream())
        dm_max = float(dm_cond.max())
        qh = opt.pair_q_host.ctypes.data_as(ctypes.c_void_p)
        bp = ctypes.cast(opt.bpcache, ctypes.c_void_p)
        vj = torch.zeros_like(dmc)
        vk = torch.zeros_like(dmc)
        jobs = []
        for cij in range(opt.ncptype):
            for ckl in range(cij + 1):
                if opt.cptype[cij][3] == 0 or opt.cptype[ckl][3] == 0:
                    continue
                shape = tuple(opt.cptype[cij][:2]) + tuple(opt.cptype[ckl][:2])
                if only is not None and shape not in (only, only[2:] + only[:2]):
                    continue
                if args.noscreen:
                    fn = lambda cij=cij, ckl=ckl: lib.BQCbuild_jk_class(
                        bp, cij, ckl, None, None, None, 1.0, _ptr(vj), _ptr(vk), _ptr(dmc), nao, 1,
                        0., 0., None, _stream())
                else:
                    fn = lambda cij=cij, ckl=ckl: lib.BQCbuild_jk_class(
                        bp, cij, ckl, _ptr(opt.pair_q), qh, _ptr(dm_cond), dm_max, _ptr(vj),
                        _ptr(vk), _ptr(dmc), nao, 1, opt.direct_scf_tol, 0., None, _stream())
                jobs.append((shape, fn))
    for rep in range(args.reps):
        res, tot = {}, 0.
        for shape, fn in jobs:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            err = fn()
            e1.record()
            torch.cuda.synchronize()
            if err:
                raise RuntimeError('J/K build failed for class %s (%d)' % (shape, err))
            ms = e0.elapsed_time(e1)
            key = '(%s%s|%s%s)' % tuple('spdf'[x] for x in shape)
            res[key] = res.get(key, 0.) + ms
            tot += ms
    print(json.dumps({'per_class': args.impl, 'workload': '(H2O)%d/%s-shaped' % (args.nwater, args.basis),
                      'density': JKPY_DENSITY, 'screen': not args.noscreen, 'total_ms': round(tot, 2),
                      'classes_ms': {k: round(v, 3) for k, v in sorted(res.items(), key=lambda x: -x[1])}}))


def max_over_ranks(value, device):
    """The largest value over the ranks of the default process group: the
    step time of N replicas is that of the slowest."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


JKPY_DENSITY = 'random symmetric AO density (rand + rand^T) x 0.1, seed 2341'


def jkpy_density(opt):
    """The density of the reference's J/K timing script (cuobc/test/jk.py),
    in the internal Cartesian basis of opt."""
    import torch
    rng = np.random.default_rng(2341)
    n0 = opt.coeff.shape[1]
    dm = rng.random((n0, n0))
    dm = torch.as_tensor(0.1 * (dm + dm.T), device='cuda')
    C = opt.coeff_dev
    return (C @ dm @ C.T)[None].contiguous()


def time_build(fn, reps=2):
    """Shortest of reps CUDA-event timed calls after one warm-up call (s)."""
    import torch
    fn()
    best = 1e30
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return best


def ctypes_peak(lib):
    import ctypes
    f = ctypes.c_double(0)
    ms = ctypes.c_float(0)
    lib.BQCfp64_fma_peak(ctypes.byref(f), ctypes.byref(ms))
    return f.value


if __name__ == '__main__':
    main()
