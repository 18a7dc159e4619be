"""Second, independent restatement of the reference encoders' core -- TEST
INFRASTRUCTURE ONLY (the tests diff it against the C++ oracle; nothing else
imports it).

Written from the Rust sources of block_compression v0.3.0 in numpy, separately
from the C++ oracle: every function works on n blocks at once, in float32
arrays, with the reference's operation order, so each element is rounded
exactly as the Rust f32 code rounds it (numpy float32 arithmetic is IEEE
binary32 with round-to-nearest-even and never fuses a multiply-add; sqrt and
division are correctly rounded). Data-dependent branches become masks.

Rust semantics restated:
  `x as i32` / `as u32`  truncation toward zero, saturating, NaN -> 0   (as_int)
  f32::min / f32::max    IEEE minNum / maxNum                            (np.fmin / np.fmax)
  f32::clamp             `if x < lo {lo}; if x > hi {hi}`, NaN passes    (clamp_f)
  i32 `/`                truncation toward zero                          (tdiv)
  `<<` on u32            high bits dropped                               (& 0xFFFFFFFF)

Blocks are planar float32 [64] (R 0..15, G 16..31, B 32..47, A 48..63), the
layout of BlockCompressorBC15 / BlockCompressorBC7 (src/encode/bc1_to_5.rs:14-40).
"""
import numpy as np

F = np.float32
U32 = 0xFFFFFFFF


def as_int(x, lo=-(2 ** 31), hi=2 ** 31 - 1):
    """Rust `as i32` (or `as u32` with lo=0, hi=2**32-1) of float32 values."""
    x = np.asarray(x, dtype=np.float64)
    t = np.trunc(np.where(np.isnan(x), 0.0, x))
    return np.clip(t, lo, hi).astype(np.int64)


def clamp_f(x, lo, hi):
    x = np.where(x < F(lo), F(lo), x)
    return np.where(x > F(hi), F(hi), x).astype(F)


def tdiv(a, b):
    """i32 division, truncating toward zero."""
    q = np.abs(a) // b
    return np.where(a < 0, -q, q)


def sq(x):
    return x * x


def planar_blocks(img):
    """(h, w, 4) uint8 -> (n, 64) float32 planar blocks, row-major block order
    (load_block_interleaved_rgba, src/encode/bc1_to_5.rs:14-40)."""
    h, w = img.shape[:2]
    t = img.reshape(h // 4, 4, w // 4, 4, 4).transpose(0, 2, 4, 1, 3)  # by, bx, channel, y, x
    return np.ascontiguousarray(t.reshape(-1, 64)).astype(F)


# ---- BC1 (src/encode/bc1_to_5.rs:157-429) ----------------------------------------------------


def _covar_dc(block):
    """compute_covar_dc (:157-192)."""
    n = block.shape[0]
    dc = []
    for p in range(3):
        acc = np.zeros(n, F)
        for k in range(16):
            acc = acc + block[:, k + p * 16]
        dc.append(acc / F(16.0))
    cov = [np.zeros(n, F) for _ in range(6)]
    for k in range(16):
        r0 = block[:, k] - dc[0]
        r1 = block[:, k + 16] - dc[1]
        r2 = block[:, k + 32] - dc[2]
        cov[0] = cov[0] + r0 * r0
        cov[1] = cov[1] + r0 * r1
        cov[2] = cov[2] + r0 * r2
        cov[3] = cov[3] + r1 * r1
        cov[4] = cov[4] + r1 * r2
        cov[5] = cov[5] + r2 * r2
    return cov, dc


def _axis3(cov, iterations):
    """ssymv + compute_axis3 (:194-223)."""
    n = cov[0].shape[0]
    a = [np.ones(n, F), np.ones(n, F), np.ones(n, F)]
    ax = a
    for i in range(iterations):
        ax = [cov[0] * a[0] + cov[1] * a[1] + cov[2] * a[2],
              cov[1] * a[0] + cov[3] * a[1] + cov[4] * a[2],
              cov[2] * a[0] + cov[4] * a[1] + cov[5] * a[2]]
        a = list(ax)
        if i % 2 == 1:
            norm_sq = F(0.0) + ax[0] * ax[0]
            norm_sq = norm_sq + ax[1] * ax[1]
            norm_sq = norm_sq + ax[2] * ax[2]
            rnorm = F(1.0) / np.sqrt(norm_sq)
            a = [v * rnorm for v in a]
    return a


def _pick_endpoints(block, axis, dc):
    """pick_endpoints (:225-256)."""
    n = block.shape[0]
    min_dot = np.full(n, 256.0 * 256.0, F)
    max_dot = np.zeros(n, F)
    for k in range(16):
        dot = F(0.0) + (block[:, k] - dc[0]) * axis[0]
        dot = dot + (block[:, 16 + k] - dc[1]) * axis[1]
        dot = dot + (block[:, 32 + k] - dc[2]) * axis[2]
        min_dot = np.fmin(min_dot, dot)
        max_dot = np.fmax(max_dot, dot)
    small = (max_dot - min_dot) < F(1.0)
    min_dot = np.where(small, min_dot - F(0.5), min_dot)
    max_dot = np.where(small, max_dot + F(0.5), max_dot)
    norm_sq = F(0.0) + axis[0] * axis[0]
    norm_sq = norm_sq + axis[1] * axis[1]
    norm_sq = norm_sq + axis[2] * axis[2]
    rnorm_sq = F(1.0) / norm_sq
    c0 = [clamp_f(dc[p] + min_dot * rnorm_sq * axis[p], 0.0, 255.0) for p in range(3)]
    c1 = [clamp_f(dc[p] + max_dot * rnorm_sq * axis[p], 0.0, 255.0) for p in range(3)]
    return c0, c1


def _dec565(p):
    """dec_rgb565 (:258-266)."""
    b5, g6, r5 = p & 31, (p >> 5) & 63, (p >> 11) & 31
    return [((r5 << 3) + (r5 >> 2)).astype(F), ((g6 << 2) + (g6 >> 4)).astype(F), ((b5 << 3) + (b5 >> 2)).astype(F)]


def _enc565(c):
    """enc_rgb565 (:268-278)."""
    r, g, b = as_int(c[0]), as_int(c[1]), as_int(c[2])
    r5 = (r * 31 + 128 + ((r * 31) >> 8)) >> 8
    g6 = (g * 63 + 128 + ((g * 63) >> 8)) >> 8
    b5 = (b * 31 + 128 + ((b * 31) >> 8)) >> 8
    return (r5 << 11) + (g6 << 5) + b5


def _fast_quant(block, p0, p1):
    """fast_quant (:280-321)."""
    c0, c1 = _dec565(p0), _dec565(p1)
    d = [c1[p] - c0[p] for p in range(3)]
    sq_norm = F(0.0) + d[0] * d[0]
    sq_norm = sq_norm + d[1] * d[1]
    sq_norm = sq_norm + d[2] * d[2]
    with np.errstate(divide="ignore", invalid="ignore"):
        rsq = F(1.0) / sq_norm
        d = [v * (rsq * F(3.0)) for v in d]
        bias = F(0.5)
        for p in range(3):
            bias = bias - c0[p] * d[p]
        bits = np.zeros(block.shape[0], np.int64)
        for k in range(16):
            dot = F(0.0) + block[:, k] * d[0]
            dot = dot + block[:, k + 16] * d[1]
            dot = dot + block[:, k + 32] * d[2]
            q = np.clip(as_int(dot + bias), 0, 3)
            bits = bits + q * (4 ** k)
    return bits & U32


def _bc1_refine(block, bits, dc):
    """bc1_refine (:323-374)."""
    n = block.shape[0]
    flat = (bits ^ ((bits * 4) & U32)) < 4
    atb1 = [np.zeros(n, F) for _ in range(3)]
    sum_q = np.zeros(n, F)
    sum_qq = np.zeros(n, F)
    sb = bits.copy()
    for k in range(16):
        q = (sb & 3).astype(F)
        sb = sb >> 2
        x = F(3.0) - q
        sum_q = sum_q + q
        sum_qq = sum_qq + q * q
        for p in range(3):
            atb1[p] = atb1[p] + x * block[:, k + p * 16]
    s = [dc[p] * F(16.0) for p in range(3)]
    atb2 = [F(3.0) * s[p] - atb1[p] for p in range(3)]
    cxx = F(144.0) - F(6.0) * sum_q + sum_qq
    cyy = sum_qq
    cxy = F(3.0) * sum_q - sum_qq
    with np.errstate(divide="ignore", invalid="ignore"):
        scale = F(3.0) * (F(1.0) / (cxx * cyy - cxy * cxy))
        c0 = [clamp_f((atb1[p] * cyy - atb2[p] * cxy) * scale, 0.0, 255.0) for p in range(3)]
        c1 = [clamp_f((atb2[p] * cxx - atb1[p] * cxy) * scale, 0.0, 255.0) for p in range(3)]
    c0 = [np.where(flat, dc[p], c0[p]) for p in range(3)]
    c1 = [np.where(flat, dc[p], c1[p]) for p in range(3)]
    return _enc565(c0), _enc565(c1)


def _fix_qbits(q):
    """fix_qbits (:376-384)."""
    q0, q1 = q & 0x55555555, q & 0xAAAAAAAA
    return ((q1 >> 1) + (q1 ^ ((q0 << 1) & U32))) & U32


def bc1_core(block):
    """compress_block_bc1_core (:386-429): (n, 64) float32 -> (n, 2) uint32."""
    block = np.asarray(block, F)
    cov, dc = _covar_dc(block)
    eps = F(np.finfo(np.float32).eps)
    cov[0] = cov[0] + eps
    cov[3] = cov[3] + eps
    cov[5] = cov[5] + eps
    axis = _axis3(cov, 4)
    c0, c1 = _pick_endpoints(block, axis, dc)
    p0, p1 = _enc565(c0), _enc565(c1)
    p0, p1 = np.maximum(p0, p1), np.minimum(p0, p1)  # swap so that p0 >= p1
    bits = _fast_quant(block, p0, p1)
    p0, p1 = _bc1_refine(block, bits, dc)
    p0, p1 = np.maximum(p0, p1), np.minimum(p0, p1)
    d0 = ((p1 << 16) | p0) & U32
    d1 = _fix_qbits(_fast_quant(block, p0, p1))
    return np.stack([d0, d1], 1).astype(np.uint32)


def bc3_alpha(block):
    """compress_block_bc3_alpha (:431-472) on block[48..64]: (n, 64) -> (n, 2) uint32."""
    block = np.asarray(block, F)
    n = block.shape[0]
    e0 = np.full(n, 255.0, F)
    e1 = np.zeros(n, F)
    for k in range(16):
        e0 = np.fmin(e0, block[:, 48 + k])
        e1 = np.fmax(e1, block[:, 48 + k])
    e1 = np.where(e0 == e1, e0 + F(0.1), e1)
    scale = F(7.0) / (e1 - e0)
    qb = [np.zeros(n, np.int64), np.zeros(n, np.int64)]
    for k in range(16):
        proj = (block[:, 48 + k] - e0) * scale + F(0.5)
        q = 7 - np.clip(as_int(proj), 0, 7)
        q = np.where(q > 0, q + 1, q)
        q = np.where(q == 8, 1, q)
        qb[k // 8] = qb[k // 8] | (q << ((k % 8) * 3))
    a0 = np.clip(as_int(e0, 0, U32), 0, 255)
    a1 = np.clip(as_int(e1, 0, U32), 0, 255)
    d0 = ((a0 << 8) | a1 | (qb[0] << 16)) & U32
    d1 = ((qb[0] >> 16) | (qb[1] << 8)) & U32
    return np.stack([d0, d1], 1).astype(np.uint32)


def compress_bc15(variant, img):
    """compress_bc1 .. compress_bc5 (src/encode.rs:259-500) of an (h, w, 4)
    uint8 image -> the packed little-endian blocks, row-major."""
    blocks = planar_blocks(img)
    n = blocks.shape[0]
    if variant == 0:
        words = bc1_core(blocks)
    elif variant == 1:  # load_block_alpha_4bit (bc1_to_5.rs:84-115) + colour
        a = (blocks[:, 48:64] / F(255.0)) * F(15.0)
        a4 = as_int(a, 0, U32)
        w0 = np.zeros(n, np.int64)
        w1 = np.zeros(n, np.int64)
        for k in range(16):
            pos = (k // 4) * 16 + (k % 4) * 4
            if pos < 32:
                w0 |= (a4[:, k] << pos) & U32
            else:
                w1 |= (a4[:, k] << (pos - 32)) & U32
        words = np.concatenate([np.stack([w0, w1], 1).astype(np.uint32), bc1_core(blocks)], 1)
    elif variant == 2:
        words = np.concatenate([bc3_alpha(blocks), bc1_core(blocks)], 1)
    elif variant == 3:  # load_block_r_8bit into slots 48..63
        r = blocks.copy()
        r[:, 48:64] = blocks[:, 0:16]
        words = bc3_alpha(r)
    elif variant == 4:
        r, g = blocks.copy(), blocks.copy()
        r[:, 48:64] = blocks[:, 0:16]
        g[:, 48:64] = blocks[:, 16:32]
        words = np.concatenate([bc3_alpha(r), bc3_alpha(g)], 1)
    else:
        raise ValueError("BC1-BC5 only")
    return np.ascontiguousarray(words.astype("<u4")).view(np.uint8).reshape(-1)


# ---- shared BPTC math (src/encode/common.rs) --------------------------------------------------

UNQUANT = {2: np.array([0, 21, 43, 64]), 3: np.array([0, 9, 18, 27, 37, 46, 55, 64]),
           4: np.array([0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64])}


def block_quant(block, bits, ep, pattern, channels):
    """block_quant (common.rs:422-481). block (n, 64), ep (n, 24) float32 (the
    subset-j pair at ep[8j .. 8j+8]), pattern (n,) uint32 (2 bits per pixel).
    Returns (qblock (n, 2) uint32, total_err (n,) float32)."""
    block = np.asarray(block, F)
    ep = np.asarray(ep, F)
    pattern = np.asarray(pattern, np.int64)
    n = block.shape[0]
    levels = 1 << bits
    table = UNQUANT[bits] if bits in (2, 3) else UNQUANT[4]
    total = np.zeros(n, F)
    qb = [np.zeros(n, np.int64), np.zeros(n, np.int64)]
    rows = np.arange(n)
    for k in range(16):
        j = (pattern >> (2 * k)) & 3
        ea = [ep[rows, 8 * j + p] for p in range(channels)]
        eb = [ep[rows, 8 * j + 4 + p] for p in range(channels)]
        proj = F(0.0)
        div = F(0.0)
        for p in range(channels):
            proj = proj + (block[:, k + p * 16] - ea[p]) * (eb[p] - ea[p])
            div = div + sq(eb[p] - ea[p])
        with np.errstate(divide="ignore", invalid="ignore"):
            proj = proj / div
            q1 = as_int(proj * F(levels) + F(0.5))
        q1c = np.clip(q1, 1, levels - 1)
        w0, w1 = table[q1c - 1], table[q1c]
        err0 = F(0.0)
        err1 = F(0.0)
        for p in range(channels):
            ia, ib = as_int(ea[p]), as_int(eb[p])
            v0 = tdiv((64 - w0) * ia + w0 * ib + 32, 64).astype(F)
            v1 = tdiv((64 - w1) * ia + w1 * ib + 32, 64).astype(F)
            err0 = err0 + sq(v0 - block[:, k + p * 16])
            err1 = err1 + sq(v1 - block[:, k + p * 16])
        take0 = err0 < err1
        best_q = np.where(take0, q1c - 1, q1c)
        qb[k // 8] = qb[k // 8] | (best_q << (4 * (k % 8)))
        total = total + np.where(take0, err0, err1)
    return np.stack(qb, 1).astype(np.uint32), total


def opt_endpoints(ep, block, bits, qblock, mask, channels):
    """opt_endpoints (common.rs:142-205): least-squares endpoints of the
    pixels in `mask` for fixed indices. ep (n, 8) float32 is updated (only
    the first `channels` of each endpoint) and returned."""
    block = np.asarray(block, F)
    ep = np.array(ep, F)
    qblock = np.asarray(qblock, np.int64)
    mask = np.asarray(mask, np.int64)
    n = block.shape[0]
    l1 = F((1 << bits) - 1)
    atb1 = [np.zeros(n, F) for _ in range(4)]
    s = [np.zeros(n, F) for _ in range(5)]
    sum_q = np.zeros(n, F)
    sum_qq = np.zeros(n, F)
    for k in range(16):
        q = ((qblock[:, k // 8] >> (4 * (k % 8))) & 15).astype(F)
        on = ((mask >> k) & 1) == 1
        x = l1 - q
        sum_q = np.where(on, sum_q + q, sum_q)
        sum_qq = np.where(on, sum_qq + q * q, sum_qq)
        s[4] = np.where(on, s[4] + F(1.0), s[4])
        for p in range(channels):
            v = block[:, k + p * 16]
            s[p] = np.where(on, s[p] + v, s[p])
            atb1[p] = np.where(on, atb1[p] + x * v, atb1[p])
    atb2 = [l1 * s[p] - atb1[p] for p in range(channels)]
    cxx = s[4] * sq(l1) - F(2.0) * l1 * sum_q + sum_qq
    cyy = sum_qq
    cxy = l1 * sum_q - sum_qq
    det = cxx * cyy - cxy * cxy
    with np.errstate(divide="ignore", invalid="ignore"):
        scale = l1 / det
        flat = np.abs(det) < F(0.001)
        for p in range(channels):
            e0 = (atb1[p] * cyy - atb2[p] * cxy) * scale
            e1 = (atb2[p] * cxx - atb1[p] * cxy) * scale
            m = s[p] / s[4]
            ep[:, p] = np.where(flat, m, e0)
            ep[:, 4 + p] = np.where(flat, m, e1)
    return ep


def _stats_masked(block, mask, channels):
    """compute_stats_masked (common.rs:294-332)."""
    n = block.shape[0]
    st = [np.zeros(n, F) for _ in range(15)]
    for k in range(16):
        flag = ((mask >> k) & 1).astype(F)
        c = [block[:, k + p * 16] * flag if p < channels else np.zeros(n, F) for p in range(4)]
        st[14] = st[14] + flag
        st[10] = st[10] + c[0]
        st[11] = st[11] + c[1]
        st[12] = st[12] + c[2]
        st[0] = st[0] + c[0] * c[0]
        st[1] = st[1] + c[0] * c[1]
        st[2] = st[2] + c[0] * c[2]
        st[4] = st[4] + c[1] * c[1]
        st[5] = st[5] + c[1] * c[2]
        st[7] = st[7] + c[2] * c[2]
        if channels == 4:
            st[13] = st[13] + c[3]
            st[3] = st[3] + c[0] * c[3]
            st[6] = st[6] + c[1] * c[3]
            st[8] = st[8] + c[2] * c[3]
            st[9] = st[9] + c[3] * c[3]
    return st


def _covar_from_stats(st, channels):
    """covar_from_stats (common.rs:334-350)."""
    n = st[0].shape[0]
    cv = [np.zeros(n, F) for _ in range(10)]
    with np.errstate(divide="ignore", invalid="ignore"):
        cv[0] = st[0] - st[10] * st[10] / st[14]
        cv[1] = st[1] - st[10] * st[11] / st[14]
        cv[2] = st[2] - st[10] * st[12] / st[14]
        cv[4] = st[4] - st[11] * st[11] / st[14]
        cv[5] = st[5] - st[11] * st[12] / st[14]
        cv[7] = st[7] - st[12] * st[12] / st[14]
        if channels == 4:
            cv[3] = st[3] - st[10] * st[13] / st[14]
            cv[6] = st[6] - st[11] * st[13] / st[14]
            cv[8] = st[8] - st[12] * st[13] / st[14]
            cv[9] = st[9] - st[13] * st[13] / st[14]
    return cv


def _ssymv(cv, b, channels):
    """ssymv3 / ssymv4 (common.rs:247-258)."""
    if channels == 3:
        return [cv[0] * b[0] + cv[1] * b[1] + cv[2] * b[2],
                cv[1] * b[0] + cv[4] * b[1] + cv[5] * b[2],
                cv[2] * b[0] + cv[5] * b[1] + cv[7] * b[2]]
    return [cv[0] * b[0] + cv[1] * b[1] + cv[2] * b[2] + cv[3] * b[3],
            cv[1] * b[0] + cv[4] * b[1] + cv[5] * b[2] + cv[6] * b[3],
            cv[2] * b[0] + cv[5] * b[1] + cv[7] * b[2] + cv[8] * b[3],
            cv[3] * b[0] + cv[6] * b[1] + cv[8] * b[2] + cv[9] * b[3]]


def _compute_axis(cv, iterations, channels):
    """compute_axis (common.rs:260-292)."""
    n = cv[0].shape[0]
    a = [np.ones(n, F) for _ in range(channels)]
    with np.errstate(divide="ignore", invalid="ignore"):
        for i in range(iterations):
            ax = _ssymv(cv, a, channels)
            a = list(ax)
            if i % 2 == 1:
                norm_sq = F(0.0)
                for p in range(channels):
                    norm_sq = norm_sq + sq(ax[p])
                rnorm = F(1.0) / np.sqrt(norm_sq)
                a = [v * rnorm for v in a]
    return a


def _pca_bound(cv, channels):
    """get_pca_bound (common.rs:208-245)."""
    inv_var = F(1.0) / (F(256.0) * F(256.0))
    c = [v * inv_var for v in cv]
    eps = F(0.001) * F(0.001)
    c[0] = c[0] + eps
    c[4] = c[4] + eps
    c[7] = c[7] + eps
    axis = _compute_axis(c, 4, channels)
    a = _ssymv(c, axis, channels)
    s = F(0.0)
    for p in range(channels):
        s = s + sq(a[p])
    lam = np.sqrt(s)
    bound = c[0] + c[4] + c[7]
    if channels == 4:
        bound = bound + c[9]
    bound = bound - lam
    return np.fmax(bound, F(0.0))


def block_pca_bound_split(block, mask, channels):
    """block_pca_bound_split (common.rs:396-420) with the whole block's
    statistics as full_stats: (n,) float32."""
    block = np.asarray(block, F)
    mask = np.asarray(mask, np.int64)
    full = _stats_masked(block, np.full(block.shape[0], 0xFFFFFFFF, np.int64), channels)
    st = _stats_masked(block, mask, channels)
    cv1 = _covar_from_stats(st, channels)
    cv2 = _covar_from_stats([full[i] - st[i] for i in range(15)], channels)
    bound = F(0.0) + _pca_bound(cv1, channels)
    bound = bound + _pca_bound(cv2, channels)
    return np.sqrt(bound) * F(256.0)


def block_segment_core(block, mask, channels):
    """block_segment_core (common.rs:483-518) with block_pca_axis (:370-394):
    (n, 8) float32 endpoints (channels beyond `channels` are 0)."""
    block = np.asarray(block, F)
    mask = np.asarray(mask, np.int64)
    n = block.shape[0]
    st = _stats_masked(block, mask, channels)
    with np.errstate(divide="ignore", invalid="ignore"):
        dc = [st[10 + p] / st[14] for p in range(channels)]
    cv = _covar_from_stats(st, channels)
    inv_var = F(1.0) / (F(256.0) * F(256.0))
    cv = [v * inv_var for v in cv]
    eps = F(0.001) * F(0.001)
    for i in (0, 4, 7, 9):
        cv[i] = cv[i] + eps
    axis = _compute_axis(cv, 8, channels)
    lo = np.full(n, np.inf, F)
    hi = np.full(n, -np.inf, F)
    for k in range(16):
        on = ((mask >> k) & 1) == 1
        dot = F(0.0)
        for p in range(channels):
            dot = dot + axis[p] * (block[:, 16 * p + k] - dc[p])
        lo = np.where(on, np.fmin(lo, dot), lo)
        hi = np.where(on, np.fmax(hi, dot), hi)
    small = (hi - lo) < F(1.0)
    lo = np.where(small, lo - F(0.5), lo)
    hi = np.where(small, hi + F(0.5), hi)
    ep = np.zeros((n, 8), F)
    for i, ext in enumerate((lo, hi)):
        for p in range(channels):
            ep[:, 4 * i + p] = ext * axis[p] + dc[p]
    return ep


# ---- BC7 endpoint quantisation (src/encode/bc7.rs:97-237) ----------------------------------------


def _unpack_to_byte(v, bits):
    vv = v << (8 - bits)
    return vv + (vv >> bits)


def _ep_quant0367(ep, mode, channels):
    bits = 4 if mode == 0 else (5 if mode == 7 else 7)
    levels2 = (1 << bits) * 2 - 1
    qep = np.zeros((ep.shape[0], 8), np.int64)
    for i in range(2):
        qb = np.zeros((ep.shape[0], 8), np.int64)
        for b in range(2):
            for p in range(4):
                v = as_int((ep[:, i * 4 + p] / F(255.0) * F(levels2) - F(b)) / F(2.0) + F(0.5)) * 2 + b
                qb[:, b * 4 + p] = np.clip(v, b, levels2 - 1 + b)
        eb = qb.astype(F)
        if mode == 0:
            eb = _unpack_to_byte(qb, 5).astype(F)
        err0 = F(0.0)
        err1 = F(0.0)
        for p in range(channels):
            err0 = err0 + sq(ep[:, i * 4 + p] - eb[:, p])
            err1 = err1 + sq(ep[:, i * 4 + p] - eb[:, 4 + p])
        first = (err0 < err1)[:, None]
        qep[:, i * 4:i * 4 + 4] = np.where(first, qb[:, 0:4], qb[:, 4:8])
    return qep


def _ep_quant1(ep):
    qb = np.zeros((ep.shape[0], 16), np.int64)
    for b in range(2):
        for i in range(8):
            v = as_int((ep[:, i] / F(255.0) * F(127.0) - F(b)) / F(2.0) + F(0.5)) * 2 + b
            qb[:, b * 8 + i] = np.clip(v, b, 126 + b)
    eb = _unpack_to_byte(qb, 7).astype(F)
    err0 = F(0.0)
    err1 = F(0.0)
    for j in range(2):
        for p in range(3):
            err0 = err0 + sq(ep[:, j * 4 + p] - eb[:, j * 4 + p])
            err1 = err1 + sq(ep[:, j * 4 + p] - eb[:, 8 + j * 4 + p])
    return np.where((err0 < err1)[:, None], qb[:, 0:8], qb[:, 8:16])


def _ep_quant245(ep, mode):
    levels = 1 << (7 if mode == 5 else 5)
    return np.clip(as_int(ep / F(255.0) * F(levels - 1) + F(0.5)), 0, levels - 1)


PAIRS = [3, 2, 3, 2, 1, 1, 1, 2]


def ep_quant_dequant(ep, mode, channels):
    """ep_quant + ep_dequant (bc7.rs:191-237): ep (n, 24) float32 ->
    (qep (n, 24) int64, dequantised ep (n, 24) float32); entries past the
    mode's pairs are returned unchanged (qep 0)."""
    ep = np.array(ep, F)
    qep = np.zeros(ep.shape, np.int64)
    for i in range(PAIRS[mode]):
        seg = ep[:, i * 8:i * 8 + 8]
        if mode in (0, 3, 6, 7):
            qep[:, i * 8:i * 8 + 8] = _ep_quant0367(seg, mode, channels)
        elif mode == 1:
            qep[:, i * 8:i * 8 + 8] = _ep_quant1(seg)
        else:
            qep[:, i * 8:i * 8 + 8] = _ep_quant245(seg, mode)
    m = 8 * PAIRS[mode]
    if mode in (3, 6):
        ep[:, :m] = qep[:, :m].astype(F)
    elif mode in (1, 5):
        ep[:, :m] = _unpack_to_byte(qep[:, :m], 7).astype(F)
    elif mode in (0, 2, 4):
        ep[:, :m] = _unpack_to_byte(qep[:, :m], 5).astype(F)
    else:
        ep[:, :m] = _unpack_to_byte(qep[:, :m], 6).astype(F)
    return qep, ep
