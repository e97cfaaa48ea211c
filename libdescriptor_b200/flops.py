"""Algorithmic FP64 operation counts per centre atom (roofline numerator).

Convention: add / mul = 1 flop, FMA = 2 flops, complex arithmetic counted as
written; each library call (exp, sincos, sqrt, divide, tan, pow, cos) costs
W_op flops, W_op measured on the device (``ld_measure_fp64_op_cost``: the
FP64-pipe flops that fit in the time of one call).  Work is counted for the
needed outputs only, along the loops of the kernels:

bispectrum (twojmax J), along the three kernels of a descriptor + VJP pass:
  U (one centre per CTA): per in-cutoff neighbour and computed left-half
    element (j, ma, mb <= j/2; the middle column's mirrored rows excluded)
    recursion b-term 8 (ma >= 1) + a-term 10 (ma < j), Utot += 4;
    calls: sqrt x2, tan, divide x2, cos (switching function)
  Z / B / Y (rows in lanes): per Z term 10 per (ma1, mb1) + 4 per ma1 row,
    for the triples the outputs (forward) or the adjoint (gradient) need;
    B 4 per element; betaj 2 per map entry; Y 4 per (element, triple)
  pair gradient (reverse mode, one (centre, neighbour) pair per slot):
    forward recompute of the recursion, 8 / 10 per element as above; the
    backward sweep per element: seed 7 (ubar += w Y, S += w Re(conj(Y) u)),
    then 20 per b-term and 20 per a-term (ubar of the two inputs, abar or
    bbar), 2 per mirrored middle-column row and per element of a born
    column (the copies reversed); per pair 24 (chain to x, y, z) + 15
    (forces) + 4 per column (column sums); calls: sqrt x2, tan, divide x5,
    sincos x2 (theta0, switching function)

symmetry functions, per listed neighbour: staging 8 + sqrt + divide + cos;
per pair output 6 + exp (g2); per triplet 25 + 2 sqrt + 3 divide + 2 cos
(fb, fd) and per three-body output 12 + one exp per distinct eta; the
gradient adds 14 per output and 60 + 3 divide per triplet.
"""
from __future__ import annotations

from functools import lru_cache

OPS = {"exp": 0, "sincos": 1, "sqrt": 2, "div": 3, "tan": 4, "pow": 5, "cos": 6}


def measure_weights(fp64_tflops: float, iters: int = 2048) -> dict:
    """W_op for every call, measured on the current device."""
    from . import _libdescriptor as _ext

    return {k: float(_ext._measure_fp64_op_cost(v, iters, fp64_tflops)) for k, v in OPS.items()}


DEFAULT_WEIGHTS = {"exp": 20.0, "sincos": 40.0, "sqrt": 12.0, "div": 12.0, "tan": 40.0,
                   "pow": 60.0, "cos": 30.0}


# per-element and per-pair FP64 flops of the bispectrum kernels' loop bodies
U_B, U_A, U_ACC = 8, 10, 4            # recursion b-term, a-term; Utot accumulation
R_SEED, R_B, R_A, R_COPY = 7, 20, 20, 2
R_PAIR, R_COL = 24 + 15, 4
Z_TERM, Z_ROW, B_EL, BETA_ENTRY, Y_EL = 10, 4, 4, 2, 4


@lru_cache(maxsize=None)
def _bs_tables(J: int, style: int):
    """(left elements with their (ma>=1, ma<j) flags, Z work, outputs, triples)."""
    elems = []
    for j in range(1, J + 1):
        h = j // 2
        for ma in range(j + 1):
            for mb in range(h + 1):
                if j % 2 == 0 and mb == h and ma > h:
                    continue
                elems.append((ma >= 1, ma < j))
    outs = []
    if style == 0:
        outs = [(a, b, c) for a in range(J + 1) for b in range(a + 1) for c in range(a - b, min(J, a + b) + 1, 2)]
    elif style == 1:
        outs = [(a, a, c) for a in range(J + 1) for c in range(0, min(J, 2 * a) + 1, 2)]
    elif style == 2:
        outs = [(a, a, a) for a in range(J + 1)]
    else:
        outs = [(a, b, c) for a in range(J + 1) for b in range(a + 1)
                for c in range(a - b, min(J, a + b) + 1, 2) if c >= a]
    trip_all = [(a, b, c) for a in range(J + 1) for b in range(a + 1) for c in range(a - b, min(J, a + b) + 1, 2)]

    def key(x, y, z):
        return (max(x, y), min(x, y), z)

    valid = set(trip_all)
    outs = [o for o in outs if o in valid]   # parity-forbidden outputs are constant zero
    need_v = set(outs)
    mentries = 0
    for (a, b, c) in outs:
        for t in (key(a, b, c), key(c, b, a), key(c, a, b)):
            need_v.add(t)
            mentries += 1

    def zwork(trips):
        terms = rows = nel = 0
        for (j1, j2, j) in trips:
            for mb in range(j // 2 + 1):
                for ma in range(j + 1):
                    if j % 2 == 0 and mb == j // 2 and ma > j // 2:
                        continue
                    na = min(j1, (2 * ma - j + j2 + j1) // 2) - max(0, (2 * ma - j - j2 + j1) // 2) + 1
                    nb = min(j1, (2 * mb - j + j2 + j1) // 2) - max(0, (2 * mb - j - j2 + j1) // 2) + 1
                    terms += max(na, 0) * max(nb, 0)
                    rows += max(na, 0)
                    nel += 1
        return terms, rows, nel

    zf = zwork(sorted(set(outs)))
    zv = zwork(sorted(need_v))
    b_elems = sum((c + 1) * (c // 2 + 1) for (_, _, c) in outs)
    y_terms = 0
    for (j1, j2, j) in sorted(need_v):
        y_terms += (j + 1) * (j // 2 + 1)
    return elems, zf, zv, b_elems, len(outs), mentries, y_terms, len(trip_all)


@lru_cache(maxsize=None)
def bs_pair_reverse_flops(J: int) -> int:
    """Flops of the reverse-mode pair kernel for one (centre, neighbour) pair,
    without its library calls: forward recompute and backward sweep over the
    left-half elements a lane column holds (the middle column's mirrored rows
    excluded), the reversed copies, and the per-pair chain to the forces."""
    f = 0
    for j in range(1, J + 1):
        h = j // 2
        for mb in range(h + 1):
            for ma in range(j + 1):
                if j % 2 == 0 and mb == h and ma > h:
                    f += R_COPY          # adjoint of the mirrored row
                    continue
                f += (U_B if ma >= 1 else 0) + (U_A if ma < j else 0)
                f += R_SEED + (R_B if ma >= 1 else 0) + (R_A if ma < j else 0)
        if j % 2 == 0 and j >= 2:
            f += R_COPY * j              # the born column's inputs, reversed
    return f + R_PAIR + R_COL * (J // 2 + 1)


def bs_flops_per_atom(J: int, style: int, n_in: float, vjp: bool, w: dict | None = None) -> float:
    """Algorithmic flops per centre with n_in in-cutoff neighbours."""
    w = w or DEFAULT_WEIGHTS
    elems, zf, zv, b_elems, nout, mentries, y_terms, _ = _bs_tables(J, style)
    u_el = sum((U_B if b else 0) + (U_A if a else 0) + U_ACC for b, a in elems)
    per_nb_fwd = u_el + 2 * w["sqrt"] + w["tan"] + 2 * w["div"] + w["cos"]
    terms, rows, _ = zv if vjp else zf
    f = n_in * per_nb_fwd + Z_TERM * terms + Z_ROW * rows + B_EL * b_elems
    if vjp:
        per_pair = bs_pair_reverse_flops(J) + 2 * w["sqrt"] + w["tan"] + 5 * w["div"] + 2 * w["sincos"]
        f += n_in * per_pair + BETA_ENTRY * mentries + Y_EL * y_terms
    return float(f)


def sf_flops_per_atom(n_neigh: float, n_pair_out: int, n_three_out: int, n_eta3: int, vjp: bool,
                      n_in_pairs: float | None = None, w: dict | None = None) -> float:
    """n_in_pairs: triplets (jj < kk) whose r_ij and r_ik are inside the cutoff
    (defaults to all n(n-1)/2)."""
    w = w or DEFAULT_WEIGHTS
    trip = n_in_pairs if n_in_pairs is not None else n_neigh * (n_neigh - 1) / 2.0
    f = n_neigh * (8 + w["sqrt"] + w["div"] + w["cos"])
    f += n_neigh * n_pair_out * (6 + w["exp"])
    f += trip * (25 + 2 * w["sqrt"] + 3 * w["div"] + 2 * w["cos"] + n_three_out * 12 + n_eta3 * w["exp"])
    if vjp:
        f += n_neigh * (n_pair_out * 8 + w["div"] + 10)
        f += trip * (n_three_out * 14 + 60 + 3 * w["div"])
    return float(f)
