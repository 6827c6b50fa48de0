"""Benchmark of the direct-SCF J/K engine on one B200 (N GPUs: replicas).

Workload (one step): a complete plain-FP64 RHF solve of (H2O)_64 in the
cc-pVTZ-shaped synthetic basis (3712 AO, s-f shells) from a SAD guess to
|Delta E| <= 1e-8 Eh, direct SCF with incremental Fock builds, Schwarz
threshold 1e-13.  ``value`` is SCF wall seconds per solve (device time with
CUDA events, setup included); ``e2e`` repeats the solve through the drop-in
host API (a host SCF loop calling get_jk with numpy arrays every cycle, the
way cuobc's RHF runs under pyscf).  The roofline object describes the
dominant J/K kernel class of one full J+K build with the converged density.

--impl reference: the CPU oracle (OpenMP C restatement of the reference's
get_jk path) on the host cores, on a bounded sample of the same workload,
projected to the workload by the algorithmic FLOP count; beside it
(``reference_gpu``) one J/K build of the workload by the reference's own GPU
kernels (oracle/_ref) on the same GPU, which the main line's ``jk_build``
repeats with this engine on the same density.

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
    p.add_argument('--account', action='store_true', help='recount the plain-SCF FLOPs')
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
        if getattr(mol, 'basis_name', '') == 'cc-pvdz':
            mf.init_guess = 'mlp'
    if host_loop:
        e = mf.kernel_hostloop()
    else:
        e = mf.kernel()
    torch.cuda.synchronize()
    return mf, e


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
        'traffic': None,
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


def scf_flops(mol, conv):
    """Algorithmic FLOPs of the J/K builds of one plain-FP64 SCF solve."""
    import torch
    from byteqc_b200.scf import hf, guess
    guess._SAD_CACHE.clear()
    mf = hf.RHF(mol)
    mf.conv_tol = conv
    acc = []
    mf.jk_hook = lambda d, fp32_below: acc.append(jk_flops(mf.opt, d))
    mf.kernel()
    return float(sum(acc)), len(acc)


def cpu_sample(args, threads):
    """Oracle J/K build of a bounded sample; returns (seconds, flops of the
    sample under the FLOP convention, description)."""
    from byteqc_b200.gto.mole import Mole
    from byteqc_b200.gto.basis import synthetic_basis
    from byteqc_b200.gto.geom import water_cluster
    from oracle import oracle
    nw = 2
    mol = Mole(water_cluster(nw, seed=0), synthetic_basis(args.basis, ['O', 'H']))
    rng = np.random.default_rng(2341)
    dm = rng.random((mol.nao, mol.nao))
    dm = dm + dm.T
    t0 = time.perf_counter()
    oracle.get_jk(mol, dm, nthreads=threads)
    t = time.perf_counter() - t0
    return t, mol, '(H2O)%d/%s-shaped, one exact J+K build (no screening), %d threads' % (
        nw, args.basis, threads)


def oracle_flops(mol):
    """Algorithmic FLOPs of the oracle's exact build (every unique quartet of
    the contracted basis, general contractions counted per column)."""
    from byteqc_b200 import flops
    ls = mol._bas[:, 1]
    npr = mol._bas[:, 2]
    nc = mol._bas[:, 3]
    nb = mol.nbas
    tot = 0.
    pairs = [(i, j) for i in range(nb) for j in range(i + 1)]
    for a, (i, j) in enumerate(pairs):
        for b in range(a + 1):
            k, l = pairs[b]
            c = nc[i] * nc[j] * nc[k] * nc[l]
            tot += c * flops.quartet_flops(ls[i], ls[j], ls[k], ls[l], npr[i] * npr[j], npr[k] * npr[l])
    return tot


def main():
    args = parse()
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))

    if args.impl == 'reference':
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        mol_full = workload(args)
        for _ in range(args.warmup):
            cpu_sample(args, threads)
        ts = []
        for _ in range(args.steps):
            t_s, mol_s, desc = cpu_sample(args, threads)
            ts.append(t_s)
        t_s = float(np.mean(ts))
        f_s = oracle_flops(mol_s)
        rate = f_s / t_s
        # project the plain-FP64 SCF of the workload: the FLOPs that the GPU
        # solve needs (same convention) at the oracle's measured rate
        key = '(H2O)%d/%s' % (args.nwater, args.basis)
        recs = json.load(open(os.path.join(ROOT, 'bench_workload_flops.json')))['workloads']
        if key not in recs:
            print(json.dumps({'impl': 'reference', 'unavailable': 'no recorded FLOP count for %s' % key}))
            return
        ref = recs[key]
        value = ref['scf_flops'] / rate
        line = {'impl': 'reference', 'metric': METRIC, 'value': round(value, 2), 'unit': 's',
                'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
                'higher_is_better': False, 'dtype': 'f64', 'data': 'synthetic',
                'config': config(args, mol_full),
                'cpu_baseline': {'value': round(value, 2), 'unit': 's', 'cores': threads,
                                 'kind': 'port', 'sample': desc + '; %.3g FLOP in %.2f s, projected '
                                 'to the %.3g FLOP of the workload SCF' % (f_s, t_s, ref['scf_flops'])},
                'e2e': {'value': round(value, 2), 'unit': 's', 'h2d_bytes_per_step': 0,
                        'd2h_bytes_per_step': 0}}
        # the reference's own GPU kernels on the same GPU, one J/K build
        try:
            line['reference_gpu'] = reference_gpu_build(mol_full)
        except Exception as exc:   # report, never fail the CPU line
            line['reference_gpu'] = {'unavailable': '%s: %s' % (type(exc).__name__, exc)}
        print(json.dumps(line))
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
                        FP32_BELOW, EARLY_TOL, '; learned guess' if mol.basis_name == 'cc-pvdz' else
                        '; SAD guess (the learned guess is trained for the cc-pVDZ shape)'),
            'config': config(args, mol), 'clocks': clk.summary(), 'gpu_launches': int(launches),
            'scf': {'energy': e, 'cycles': mf.cycles, 'converged': bool(mf.converged),
                    'jk_s': round(mf.timings.get('jk', 0), 3)}}

    if not args.no_extras and rank == 0:
        # the plain FP64 form on the same GPU, same workload
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        mf_p, e_p = scf_once(mol, args.conv)
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
        # one J/K build on the density of the reference's timing script (the
        # reference arm times its own kernels on the same one)
        opt = mf.opt
        dmc = jkpy_density(opt)
        line['jk_build'] = {'s': round(time_build(lambda: opt.jk_cart(dmc)), 3),
                            'density': JKPY_DENSITY, 'tol': opt.direct_scf_tol}
        # FLOPs of the J/K builds of a plain-FP64 solve: the CPU projection's
        # numerator (recorded per workload; --account recounts on the device)
        key = '(H2O)%d/%s' % (args.nwater, args.basis)
        recs = json.load(open(os.path.join(ROOT, 'bench_workload_flops.json')))['workloads']
        if args.account or key not in recs:
            f_scf, nbuild = scf_flops(mol, args.conv)
            line['scf']['jk_builds_counted'] = nbuild
        else:
            f_scf = recs[key]['scf_flops']
        line['scf']['plain_jk_flops'] = f_scf
        line['scf']['plain_jk_tflops'] = round(f_scf / max(mf_p.timings.get('jk', 1e-9), 1e-9) / 1e12, 3)
        ref = {'scf_flops': f_scf}
        threads = os.cpu_count() or 1
        t_s, mol_s, desc = cpu_sample(args, threads)
        f_s = oracle_flops(mol_s)
        cpu_val = ref['scf_flops'] / (f_s / t_s)
        line['cpu_baseline'] = {'value': round(cpu_val, 2), 'unit': 's', 'cores': threads,
                                'kind': 'port', 'sample': desc + '; %.3g FLOP in %.2f s, projected '
                                'to the %.3g FLOP of the workload SCF' % (f_s, t_s, ref['scf_flops'])}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


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


def reference_gpu_build(mol):
    """Seconds of one J/K build by the reference's own GPU kernels (oracle/_ref,
    compiled from cuobc/lib for sm_100a) on the jk.py density, or a reason."""
    import torch
    from oracle import ref_gpu
    if not torch.cuda.is_available():
        return {'unavailable': 'no GPU'}
    if not ref_gpu.available():
        return {'unavailable': 'oracle/_ref not built (the reference sources were absent at build time)'}
    from byteqc_b200.scf import hf
    opt = hf._VHFOpt(mol).build()
    ref = ref_gpu.RefJK(opt)
    dmc = jkpy_density(opt)
    tasks = ref.tasks(dmc)
    t = time_build(lambda: ref.jk_cart(dmc, tasks=tasks), reps=1)
    ref.close()
    return {'jk_build_s': round(t, 3), 'density': JKPY_DENSITY, 'launches': len(tasks),
            'what': 'GINTbuild_jk of the reference (cuobc/lib/gvhf, cuobc/lib/gint) built for '
                    'sm_100a, driven by the restated host logic of cuobc/scf/hf.py get_jk '
                    '(log-q bins, class-level density screen); same B200, CUDA events'}


def ctypes_peak(lib):
    import ctypes
    f = ctypes.c_double(0)
    ms = ctypes.c_float(0)
    lib.BQCfp64_fma_peak(ctypes.byref(f), ctypes.byref(ms))
    return f.value


if __name__ == '__main__':
    main()
