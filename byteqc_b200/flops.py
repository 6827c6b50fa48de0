"""Algorithmic FLOP count of a J/K build (one convention for every form).

For a shell-quartet class canonicalised so that li >= lj and lk >= ll, with
L = li+lj+lk+ll, n = L//2 + 1 Rys roots, lij = li+lj, lkl = lk+ll and
nf = prod over the four shells of (l+1)(l+2)/2 Cartesian components:

  F_prim = n * [ 3*5*(lij+1)(lkl+1)                              (VRR)
               + 3*2*( sum_{t=1..lj} (lij-t+1)(lkl+1)
                     + sum_{t=1..ll} (lkl-t+1)(li+1)(lj+1) )      (HRR)
               + 3*nf ]                                           (x*y*z product, accumulate)
           + 30                                                   (pair set-up, roots amortised)
  F_dig  = 12 * nf * n_dm      (J_ij, J_kl, K_ik, K_il, K_jk, K_jl; 2 flops each)

and a build costs  sum over surviving quartets of nprim_ij*nprim_kl*F_prim + F_dig,
the surviving quartets being those that pass the plain-FP64 screening at the
same threshold (so a faster form shows up as time, not as fewer flops).
"""


def ncart(l):
    return (l + 1) * (l + 2) // 2


def f_prim(li, lj, lk, ll):
    if li < lj:
        li, lj = lj, li
    if lk < ll:
        lk, ll = ll, lk
    L = li + lj + lk + ll
    n = L // 2 + 1
    lij, lkl = li + lj, lk + ll
    nf = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    vrr = 3 * 5 * (lij + 1) * (lkl + 1)
    hrr = 3 * 2 * (sum((lij - t + 1) * (lkl + 1) for t in range(1, lj + 1)) +
                   sum((lkl - t + 1) * (li + 1) * (lj + 1) for t in range(1, ll + 1)))
    return n * (vrr + hrr + 3 * nf) + 30


def f_dig(li, lj, lk, ll, n_dm=1):
    return 12 * ncart(li) * ncart(lj) * ncart(lk) * ncart(ll) * n_dm


def quartet_flops(li, lj, lk, ll, nprim_ij, nprim_kl, n_dm=1):
    return nprim_ij * nprim_kl * f_prim(li, lj, lk, ll) + f_dig(li, lj, lk, ll, n_dm)
