"""Algorithmic work of one conversion: FP64 operations and compulsory bytes, pass by pass.

The operation counts follow the reference's operation sequence (HongYue1/KBSRC src/dsp/fft.hpp,
src/dsp/double_double.hpp, src/dsp/simd.hpp, src/resampler.cpp:34-88), counted as FP64 instructions: an add,
subtract, multiply or fused multiply-add each count 1; sign flips count 0. In these units:
  f64 add/mul 1; dd short add 11; dd accurate add 20; dd product 9 (one of them an fma); qts renormalisation 3.
This is the work any implementation of the same rounding must do; the GPU engine does exactly this per output
value (except fast's spectrum bins, which it evaluates twice).
"""
import math

SHORT, ACCURATE, F64 = "short", "accurate", "f64"
ADD = {SHORT: 11, ACCURATE: 20, F64: 1}
MUL = {SHORT: 9, ACCURATE: 9, F64: 1}


def radices(n):
    rs, t = [], n
    while t % 4 == 0:
        rs.append(4)
        t //= 4
    while t % 2 == 0:
        rs.append(2)
        t //= 2
    for p in (3, 5, 7):
        while t % p == 0:
            rs.append(p)
            t //= p
    if t != 1:
        raise ValueError("not 7-smooth")
    return rs


def cx_add(a):
    return 2 * ADD[a]


def cx_mul(a):
    return 4 * MUL[a] + 2 * ADD[a]


def stockham_ops(n, a):
    """FP64 ops of one Stockham transform of n points in arithmetic a (fft.hpp:62-151)."""
    ops, s, rem = 0, 1, n
    for r in radices(n):
        m = rem // r
        bf, bf_tw = m * s, (m - 1) * s  # butterflies, and those with stage twiddles (p != 0)
        if r == 4:
            ops += bf * 8 * cx_add(a) + bf_tw * 3 * cx_mul(a)
        elif r == 2:
            ops += bf * 2 * cx_add(a) + bf_tw * cx_mul(a)
        else:
            H = (r - 1) // 2
            per = 3 * H * cx_add(a) + H * (H * (4 * MUL[a] + 4 * ADD[a]) + 2 * cx_add(a))
            ops += bf * per + bf_tw * 2 * H * cx_mul(a)
        rem //= r
        s *= r
    return ops


def cfft_passes(h, exact, design=False):
    """Per-pass FP64 ops of the complex FFT of h points: dict with 'A' (column or direct) and 'B' (row)."""
    if not design and not exact:
        sub, sc, lanes, renorm = F64, F64, True, False
    elif design:
        sub, sc, lanes, renorm = ACCURATE, ACCURATE, False, False
    else:
        sub, sc, lanes, renorm = SHORT, ACCURATE, True, True
    if h <= 2048:
        return {"A": stockham_ops(h, sc), "B": 0, "four": False}
    N1 = max(d for d in range(1, int(math.isqrt(h)) + 1) if h % d == 0)
    N2 = h // N1
    if N1 < 8:
        return {"A": stockham_ops(h, sc), "B": 0, "four": False}
    tw = (N1 - 1) * (N2 if lanes else N2 - 1)
    rn = 6 * h if renorm else 0  # qts of re and im on every stored value
    A = N2 * stockham_ops(N1, sub) + tw * cx_mul(sub) + rn
    B = N1 * stockham_ops(N2, sub) + rn
    return {"A": A, "B": B, "four": True, "N1": N1, "N2": N2}


def task_ops(Nb, Mb, up, exact, hop, P):
    """FP64 ops of one (channel, block) task by pass: fwd_column, fwd_row, split, merge, inv_column, inv_row."""
    a = ACCURATE if exact else F64
    hf, hi = Nb // 2, Mb // 2
    fw, iv = cfft_passes(hf, exact), cfft_passes(hi, exact)
    # forward split (fft.hpp:365-408): k = 0 two adds; each k >= 1 (or each pair in dd)
    per_k = 2 * cx_add(a) + cx_mul(a) + cx_add(a) + 2 * MUL[a]
    if exact:
        pairs = hf // 2
        split = 2 * ADD[a] + pairs * per_k + (pairs - (1 if hf % 2 == 0 else 0)) * (cx_mul(a) + cx_add(a) + 2 * MUL[a])
    else:
        split = 2 * ADD[a] + (hf - 1) * per_k
    # spectrum (resampler.cpp:64-78) + inverse merge (fft.hpp:412-458)
    K = hi + 1
    if up:
        spec = K * 2 * MUL[a]
    else:
        jmax = min(hf, Mb - 1)
        folds = max(0, jmax - K + 1)
        spec = K * 2 * MUL[a] + folds * (2 * MUL[a] + cx_add(a)) + 2 * MUL[a]  # Y[Mb/2] recomputed
    per_merge = 2 * cx_add(a) + cx_mul(a) + 2 * ADD[a]
    if exact:
        pairs = hi // 2
        partners = pairs - (1 if hi % 2 == 0 else 0)
        merge = per_merge * (pairs + 1) + partners * (cx_mul(a) + 2 * ADD[a])
    else:
        merge = per_merge * hi
    out = hop * P if exact else 0  # hi + lo of every kept sample
    return {"fwd_column": fw["A"], "fwd_row": fw["B"], "split": split, "merge": spec + merge,
            "inv_column": iv["A"], "inv_row": iv["B"] + out}


def conversion_work(plan, channels, exact):
    """Totals for a plan dict (kbsrc_b200.plan keys): FP64 ops per pass and in all, compulsory HBM bytes."""
    tasks = channels * plan["nblk"]
    per = task_ops(plan["Nb"], plan["Mb"], plan["up"], exact, plan["hop"], plan["P"])
    total = {k: v * tasks for k, v in per.items()}
    # compulsory bytes: each block reads its input span (halo included) and writes its kept output
    bytes_ = tasks * 8 * (plan["Nb"] + plan["hop"] * plan["P"])
    return {"tasks": tasks, "ops_per_task": per, "ops": total, "ops_total": sum(total.values()),
            "compulsory_bytes": bytes_}


def pass_bytes(plan, exact):
    """Bytes each pass must move per task (its inputs and outputs; complex dd 32 B, f64 16 B). In float64 the split,
    spectrum and merge are one pass timed as "merge" (it reads Z, e*hf, and writes the inverse input, e*hi)."""
    e = 32 if exact else 16
    hf, hi = plan["Nb"] // 2, plan["Mb"] // 2
    four_f, four_i = hf > 2048, hi > 2048
    out = 8 * plan["hop"] * plan["P"]
    return {"fwd_column": 8 * plan["Nb"] + e * hf,
            "fwd_row": 2 * e * hf if four_f else 0,
            "split": e * hf + e * (hf + 1),
            "merge": e * (hf + 1) + e * hi if exact else e * hf + e * hi,
            "inv_column": 2 * e * hi if four_i else e * hi + out,
            "inv_row": e * hi + out if four_i else 0}


# ---------------------------------------------------------------------------------------------------------------
# split-precision form: tensor-core work (mirrors the planner of kbsrc_b200/csrc/engine.cu, make_tc_fft)
# ---------------------------------------------------------------------------------------------------------------
TC_DIGITS, TC_ACC, TC_ROWS = 7, 8, 128
TC_PRODUCTS = sum(1 for a in range(TC_DIGITS) for b in range(TC_DIGITS) if a + b < TC_ACC)  # 34
# issued accumulator blocks: data slice ta against matrix slices 0..7-ta (the eighth one zero) in wide MMAs
TC_ISSUED = sum(TC_ACC - ta for ta in range(TC_DIGITS))  # 35


def tc_factor(N):
    """(Ra, Rb) with Ra * Rb = N, both in [2, 32], Ra the largest such divisor <= sqrt(N); (N, 1) for a prime N of
    at most 32; None if there is neither."""
    best = 0
    a = 2
    while a <= 32 and a * a <= N:
        if N % a == 0 and N // a <= 32:
            best = a
        a += 1
    if best:
        return best, N // best
    return (N, 1) if 2 <= N <= 32 else None


def tc_factor3(N):
    """(Ra, Rb, Rc) with Ra * Rb * Rc = N, each <= 32 and >= N / 128, the smallest radix as large as possible; None
    if there is none."""
    lo = max(2, -(-N // TC_ROWS))
    best = None
    for a in range(lo, 33):
        if N % a:
            continue
        for b in range(a, 33):
            if (N // a) % b:
                continue
            c = N // a // b
            if b <= c <= 32 and (best is None or a > best[0]):
                best = (a, b, c)
    return best


def tc_radices(N):
    """The radices of a split-form sub-FFT of N points: two where possible, else three."""
    return tc_factor(N) or tc_factor3(N)


def tc_split(n):
    """(N1, N2): one direct sub-FFT (N2 = 1) up to 1024 points, else the four-step split nearest sqrt(n); sub-FFTs
    of two radices where any split allows them, else of three."""
    for ok in (tc_factor, tc_radices):
        if n <= 1024 and ok(n):
            return n, 1
        N1 = int(math.isqrt(n)) + 1
        while N1 >= 2:
            if N1 * N1 <= n and n % N1 == 0 and n // N1 <= 1024 and ok(N1) and ok(n // N1):
                return N1, n // N1
            N1 -= 1
    return None


def _kh(R):
    return 16 if R <= 16 else 32


def _nh(R):
    return 16 if R <= 16 else 24 if R <= 24 else 32


def _tc_stage_ops(R, eb=1):
    """Issued tensor-core operations (M x N x K x 2, padding included) of one stage of radix R."""
    if R <= 1:
        return 0
    return TC_ISSUED * 2 * TC_ROWS * 2 * _nh(R) * 2 * _kh(R)


def _tc_smem(rads, N, eb=1):
    al = lambda v: (v + 127) // 128 * 128
    rr = [R for R in rads if R > 1]
    kpad = 2 * max(_kh(R) for R in rr) * eb
    bm = lambda R: (TC_DIGITS + 1) * 2 * _nh(R) * 2 * _kh(R) * eb
    ntw = N + (rads[1] * rads[2] if len(rads) == 3 else 0)
    return al(TC_DIGITS * TC_ROWS * kpad) + sum(al(bm(R)) for R in rr) + al(ntw * 16) + al(TC_ROWS * 4) + 128


def _tc_sub_ops(N, count, eb=1):
    rads = tc_radices(N)
    F = max(1, min(TC_ROWS // (N // min(R for R in rads if R > 1)), count))
    while F > 1 and 2 * N * F * 16 + _tc_smem(rads, N, eb) > 227 * 1024:
        F -= 1
    items = -(-count // F)
    return items * sum(_tc_stage_ops(R, eb) for R in rads)


def split_work(plan, channels, eb=1):
    """Issued tensor-core operations (int8 for eb = 1, f16 for eb = 2) per task of each split-form pass, and in
    all."""
    tasks = channels * plan["nblk"]
    per = {}
    for pre, n in (("fwd", plan["Nb"] // 2), ("inv", plan["Mb"] // 2)):
        N1, N2 = tc_split(n)
        per[pre + "_column"] = _tc_sub_ops(N1, N2, eb)
        per[pre + "_row"] = _tc_sub_ops(N2, N1, eb) if N2 > 1 else 0
    return {"tasks": tasks, "int8_ops_per_task": per, "int8_ops_total": sum(per.values()) * tasks,
            "ops_per_task": per, "ops_total": sum(per.values()) * tasks}


def error_stats(y, ref):
    """Error of y against ref (the exact output): max and RMS of |y - ref| absolute, in dB of full scale 1.0, and in
    float64 ULPs of each ref sample (samples below 2^-10 of the peak left out of the ULP figures)."""
    import numpy as np
    d = np.abs(np.asarray(y, dtype=np.float64) - ref)
    mx, rms = float(d.max(initial=0.0)), float(np.sqrt(np.mean(d * d))) if d.size else 0.0
    big = np.abs(ref) >= np.abs(ref).max(initial=0.0) * 2.0 ** -10
    u = d[big] / np.spacing(np.abs(ref[big]))
    db = lambda v: round(20 * np.log10(v), 2) if v > 0 else None
    return {"max_abs": mx, "rms_abs": rms, "max_db": db(mx), "rms_db": db(rms),
            "max_ulps": float(u.max(initial=0.0)), "rms_ulps": float(np.sqrt(np.mean(u * u))) if u.size else 0.0}
