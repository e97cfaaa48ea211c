"""CPU: the index arithmetic that the GPU kernels' schedules rely on, restated
loop for loop in Python and checked exhaustively over small sizes.

* Symmetry-function triplet pairing (ld_sf.cu, ld_sfg.cu): lane l owns
  neighbour jj = l (+32, ...) and at step dd takes (jj, (jj + dd) mod n),
  dd = 1 .. n/2, the last step of an even n only for jj < n/2.  Every
  unordered pair must come exactly once, and within one step the lanes'
  second neighbours must be distinct (their gradients are then plain
  read-modify-writes, no atomics).
* Rows-in-lanes Z of the bispectrum (ld_bs2_impl.cuh, bsZ_kernel): the
  window over u_{j1} with rotating registers, the per-triple column weights
  G[mb][q] and the zero guards around the U block.  With arbitrary weights in
  place of the Clebsch-Gordan table the model must equal the direct double
  sum Z(ma, mb) = sum w(ma1, ma2) w(mb1, mb2) u1(ma1, mb1) u2(ma2, mb2), and
  every read must stay inside guard + U + guard even when the guards and the
  rest of the block hold non-zero values.
* The U-only per-centre kernel's output (bsA_kernel UOUT): each left-half
  element, its inversion image and the middle column's mirrored lower rows
  must write every element of the full U exactly once, with the right
  values.
"""
import numpy as np
import pytest


# ------------------------------------------------------- triplet pairing
def _cyclic_steps(n):
    """Per chunk of 32 lanes and step: list of (jj, kk) the lanes take."""
    dmax, dlast = (n - 1) // 2, n // 2
    steps = []
    for m0 in range(0, n, 32):
        for dd in range(1, dlast + 1):
            pairs = []
            for lane in range(32):
                jj = m0 + lane
                if jj >= n or not (dd <= dmax or jj < dlast):
                    continue
                pairs.append((jj, (jj + dd) % n))
            steps.append(pairs)
    return steps


@pytest.mark.parametrize("n", list(range(0, 71)) + [96, 97, 128])
def test_cyclic_pairing_covers_each_pair_once_with_distinct_kk(n):
    seen = {}
    for pairs in _cyclic_steps(n):
        kks = [kk for _, kk in pairs]
        assert len(kks) == len(set(kks)), (n, pairs)
        for jj, kk in pairs:
            assert jj != kk
            key = (min(jj, kk), max(jj, kk))
            seen[key] = seen.get(key, 0) + 1
    assert len(seen) == n * (n - 1) // 2
    assert all(v == 1 for v in seen.values())


# ------------------------------------------------------ rows-in-lanes Z
def _inversion_symmetric_u(J, rng):
    U = []
    for j in range(J + 1):
        a = rng.normal(size=(j + 1, j + 1)) + 1j * rng.normal(size=(j + 1, j + 1))
        for m in range(j + 1):
            for k in range(j + 1):
                if (m, k) < (j - m, j - k):
                    a[j - m, j - k] = (-1) ** (m - k) * np.conj(a[m, k])
                elif (m, k) == (j - m, j - k):
                    a[m, k] = a[m, k].real if (m - k) % 2 == 0 else 1j * a[m, k].imag
        U.append(a)
    return U


@pytest.mark.parametrize("J", [0, 1, 2, 5, 8])
def test_rows_in_lanes_z_window_equals_direct_sum(J):
    rng = np.random.default_rng(J)
    U = _inversion_symmetric_u(J, rng)
    ublock = [0]
    for j in range(J + 1):
        ublock.append(ublock[-1] + (j + 1) ** 2)
    nU = ublock[-1]
    glo, ghi = J + 1, J // 2 + 1
    # guards and block filled with finite non-zero values: a read outside a
    # row must meet a zero weight, not a zero value
    mem = rng.normal(size=glo + nU + ghi) + 1j * rng.normal(size=glo + nU + ghi)
    for j in range(J + 1):
        mem[glo + ublock[j]:glo + ublock[j + 1]] = U[j].ravel()

    def ld(e):
        assert 0 <= glo + e < len(mem), ("read outside guard + U + guard", e)
        return mem[glo + e]

    trips = [(j1, j2, j) for j1 in range(J + 1) for j2 in range(j1 + 1)
             for j in range(j1 - j2, min(J, j1 + j2) + 1, 2)]
    for (j1, j2, j) in trips:
        c, nc = (j1 + j2 - j) // 2, j // 2 + 1
        w = rng.normal(size=(j1 + 1, j2 + 1))       # stands in for cg(j1, j2, j)
        nst = min(j2, c + nc - 1) + 1
        G = np.zeros((nst, nc))
        for mb in range(nst):
            for q in range(nc):
                mb1 = c + q - mb
                if 0 <= mb1 <= j1:
                    G[mb, q] = w[mb1, mb]
        for ma in range(j + 1):
            z = np.zeros(nc, complex)
            ca = c + ma
            hi = nst - 1
            nmain = min(c, hi) + 1        # steps 0..min(c, hi): any column may be valid
            rem = nmain % nc
            for ma2 in range(max(0, ca - j1), min(j2, ca) + 1):
                ma1 = ca - ma2
                ga = w[ma1, ma2]
                xrow = ublock[j2] + ma2 * (j2 + 1)
                wrow = ublock[j1] + ma1 * (j1 + 1) + c - 1
                win = [ga * ld(wrow + q + 1) for q in range(nc)]
                for mb in range(rem):                      # shifting steps
                    x = ld(xrow + mb)
                    z += G[mb] * x * np.array(win)
                    win = [ga * ld(wrow - mb)] + win[:-1]
                for mb0 in range(rem, nmain, nc):          # rotation blocks
                    for s in range(nc):
                        mb = mb0 + s
                        x = ld(xrow + mb)
                        for q in range(nc):
                            z[q] += G[mb, q] * x * win[(q - s + nc) % nc]
                        win[(nc - 1 - s) % nc] = ga * ld(wrow - mb)
                for k in range(1, nc):                     # tail: steps c + k, columns q >= k
                    mb = c + k
                    if mb > hi:
                        break
                    x = ld(xrow + mb)
                    s = k - 1
                    for q in range(k, nc):
                        z[q] += G[mb, q] * x * win[(q - s + nc) % nc]
                    # the entering element (column 0) is never used again
            for q in range(nc):
                ref = 0j
                for ma1 in range(j1 + 1):
                    ma2 = ca - ma1
                    if not 0 <= ma2 <= j2:
                        continue
                    for mb1 in range(j1 + 1):
                        mb2 = c + q - mb1
                        if 0 <= mb2 <= j2:
                            ref += w[ma1, ma2] * w[mb1, mb2] * U[j1][ma1, mb1] * U[j2][ma2, mb2]
                assert abs(z[q] - ref) <= 1e-12 * (1 + abs(ref)), (j1, j2, j, ma, q)


# ------------------------------------------------- U-only output writer
@pytest.mark.parametrize("J", list(range(0, 11)))
def test_u_only_writer_fills_full_u_once(J):
    rng = np.random.default_rng(100 + J)
    U = _inversion_symmetric_u(J, rng)
    wself = 1.0
    ublock = [0]
    for j in range(J + 1):
        ublock.append(ublock[-1] + (j + 1) ** 2)
    out = np.full(ublock[-1], np.nan, complex)
    count = np.zeros(ublock[-1], int)
    for jl in range(J + 1):
        hj = jl // 2
        for ma in range(jl + 1):
            for m2 in range(hj + 1):                 # the left half, middle column whole
                mir = jl % 2 == 0 and m2 == hj and ma > hj
                if mir:                              # lower middle rows: mirror of row jl - ma
                    v = U[jl][jl - ma, hj]
                    sg = -1.0 if (ma - hj) & 1 else 1.0
                    v = complex(sg * v.real, -sg * v.imag)
                else:
                    v = U[jl][ma, m2] + (wself if ma == m2 else 0.0)
                k = ublock[jl] + ma * (jl + 1) + m2
                out[k] = v
                count[k] += 1
                if jl - m2 > hj:                     # inversion image in the right half
                    sg = -1.0 if (ma - m2) & 1 else 1.0
                    k = ublock[jl] + (jl - ma) * (jl + 1) + (jl - m2)
                    out[k] = complex(sg * v.real, -sg * v.imag)
                    count[k] += 1
    ref = np.concatenate([(U[j] + wself * np.eye(j + 1)).ravel() for j in range(J + 1)])
    assert (count == 1).all()
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-14)


# ----------------------------------------------- roofline flop count
W_MEASURED = {"exp": 41.2, "sincos": 89.2, "sqrt": 30.8, "div": 35.0, "tan": 89.9, "pow": 279.3, "cos": 74.9}


@pytest.mark.parametrize("J", [2, 4, 6, 8])
def test_pair_kernel_flop_count_walks_its_loops(J):
    """The reverse-mode pair kernel (bsR_kernel): lane column mb runs layers
    max(1, 2 mb) .. J forward (rev_fwd) and back (rev_bwd); per computed row
    the recursion, the seed and the backward step; mirrored middle-column
    rows only reverse their copy; at each even layer j the lane of column
    j/2 - 1 takes back the j inputs it lent to the born column."""
    from libdescriptor_b200 import flops as F

    f = 0
    for mb in range(J // 2 + 1):
        for j in range(max(1, 2 * mb), J + 1):
            h = j // 2
            middle = j % 2 == 0 and mb == h
            for ma in range(j + 1):
                if middle and ma > h:
                    f += F.R_COPY
                    continue
                b, a = ma >= 1, ma < j
                f += F.U_B * b + F.U_A * a                    # forward recompute
                f += F.R_SEED + F.R_B * b + F.R_A * a         # backward
            if j % 2 == 0 and mb == h - 1:
                f += F.R_COPY * j                             # birth of column h, reversed
    f += F.R_PAIR + F.R_COL * (J // 2 + 1)
    assert F.bs_pair_reverse_flops(J) == f


def test_bispectrum_flops_per_atom_pinned():
    """The per-atom count the benchmark's roofline divides by: 2J = 8,
    style 3, 25 in-cutoff neighbours, descriptors + VJP, the call weights
    measured on a B200 (FP64 flops in the time of one call)."""
    from libdescriptor_b200 import flops as F

    per_atom = F.bs_flops_per_atom(8, 3, 25.0, True, W_MEASURED)
    assert abs(per_atom - 727777.5) < 1.0
    # no forward-mode tangents: the gradient's per-neighbour work is the
    # reverse sweep, under three times the forward recursion's 3.1 k flops
    per_nb = F.bs_flops_per_atom(8, 3, 1.0, True, W_MEASURED) - F.bs_flops_per_atom(8, 3, 0.0, True, W_MEASURED)
    fwd_nb = F.bs_flops_per_atom(8, 3, 1.0, False, W_MEASURED) - F.bs_flops_per_atom(8, 3, 0.0, False, W_MEASURED)
    assert per_nb < 4 * fwd_nb


# ------------------------------------------- warp-per-centre U kernel
def _lblock(j):
    return sum((jj + 1) * (jj // 2 + 1) for jj in range(j))


@pytest.mark.parametrize("J", [0, 1, 2, 3, 4, 5, 6, 7, 8])
def test_warp_u_slot_reduction_covers_the_left_half(J):
    """bsU_kernel: lane (slot, mb) puts its column's sums of every layer j >=
    2 mb into the slot's row of the buffer at e = lblock(j) + ma (j/2+1) + mb,
    the middle column's mirrored rows left out; over the lanes of one slot
    every other left-half element is written exactly once, and the padded
    per-slot stride (= NC mod 16 doubles) sends a half-warp's 16 lanes to 16
    different banks for every (j, ma) they write together."""
    NC = J // 2 + 1
    SL = 32 // NC
    nL = _lblock(J + 1)
    RS = nL + ((NC - nL) % 16 + 16) % 16
    assert RS >= nL and RS % 16 == NC % 16
    seen = {}
    for mb in range(NC):
        for j in range(J + 1):
            h = j // 2
            if mb > h:
                continue
            for ma in range(j + 1):
                if j % 2 == 0 and ma > h and mb == h:
                    continue
                e = _lblock(j) + ma * (h + 1) + mb
                assert 0 <= e < nL
                seen[e] = seen.get(e, 0) + 1
    mirrors = sum(j // 2 for j in range(0, J + 1, 2))
    assert len(seen) == nL - mirrors and all(v == 1 for v in seen.values())
    for j in range(J + 1):
        h = j // 2
        for ma in range(j + 1):
            for half in (0, 16):
                banks = []
                for lane in range(half, half + 16):
                    slot, mb = divmod(lane, NC)
                    if slot >= SL or mb > h or (j % 2 == 0 and ma > h and mb == h):
                        continue
                    banks.append((slot * RS + _lblock(j) + ma * (h + 1) + mb) % 16)
                assert len(banks) == len(set(banks))


# ------------------------------------------- pair kernel row search
def _warp_search(off, n_rows, q0):
    """bsR_kernel's 32-ary search, lane by lane."""
    lo, hi = 0, n_rows - 1
    rounds = 0
    while hi > lo:
        span = hi - lo
        pos = [lo + (span * (lane + 1) + 31) // 32 for lane in range(32)]
        le = [off[p] <= q0 for p in pos]
        assert all(le[i] >= le[i + 1] for i in range(31)), "ballot not a prefix"
        k = max((i for i in range(32) if le[i]), default=-1)
        nlo = pos[k] if k >= 0 else lo
        nhi = pos[k + 1] - 1 if k < 31 else hi
        assert nlo <= nhi
        lo, hi = nlo, nhi
        rounds += 1
    return lo, rounds


@pytest.mark.parametrize("seed", range(6))
def test_pair_kernel_row_search_finds_the_last_row_at_or_below(seed):
    """The warp's first pair q0 lies in row r with off[r] <= q0 < off[r+1]
    (rows without neighbours share their offset with the next row: the last
    such row is the one that holds the pair); each slot then steps forward."""
    rng = np.random.default_rng(seed)
    n_rows = int(rng.integers(1, 40000))
    counts = rng.integers(0, 40, n_rows)
    counts[rng.random(n_rows) < 0.1] = 0
    off = np.concatenate([[0], np.cumsum(counts)])
    n_pairs = int(off[-1])
    if n_pairs == 0:
        return
    for q0 in list(rng.integers(0, n_pairs, 200)) + [0, n_pairs - 1]:
        row, rounds = _warp_search(off, n_rows, int(q0))
        want = int(np.searchsorted(off, q0, side="right")) - 1
        assert row == want and off[row] <= q0 < off[row + 1]
        assert rounds <= 4
        for slot in range(6):
            qp = int(q0) + slot
            if qp >= n_pairs:
                break
            r = row
            while r + 1 < n_rows and off[r + 1] <= qp:
                r += 1
            assert off[r] <= qp < off[r + 1]
