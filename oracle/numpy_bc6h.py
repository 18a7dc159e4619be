"""Second, independent restatement of the reference BC6H encoder -- TEST
INFRASTRUCTURE ONLY (the tests diff it against the C++ oracle; nothing else
imports it).

Written in numpy from the Rust of block_compression v0.3.0
(src/encode/bc6h.rs and the BC6H driver of src/encode.rs:590-620),
separately from the C++ oracle, for the RGBA16F input (compress_rgba16): every
step runs on all blocks at once in float32 / integer arrays with the
reference's operation order; per-block state (mode, endpoint bits,
quantisation bounds) is an array, and per-block decisions are masks. The
float primitives are those of numpy_restatement.py and the BPTC coding
helpers those of numpy_bc7.py (both also restated from the Rust).
Settings: the u32 list of BC6HSettings' #[repr(C)] fields (slow_mode,
fast_mode, refine_iterations_1p, refine_iterations_2p, fast_skip_threshold).
"""
import numpy as np

from . import numpy_bc7 as b7
from . import numpy_restatement as nr

F = np.float32
U32 = 0xFFFFFFFF
INF = F(np.inf)

# bc6h.rs:131-164 (the spans are f32 constant expressions)
PREFIX = [0, 1, 2, 6, 10, 14, 18, 22, 26, 30, 3, 7, 11, 15]
SPAN = {0: F(0.9) * F(65535.0) / F(64.0), 1: F(0.9) * F(65535.0) / F(4.0), 2: F(0.8) * F(65535.0) / F(256.0),
        5: F(0.9) * F(65535.0) / F(32.0), 6: F(0.9) * F(65535.0) / F(16.0), 9: F(65535.0), 10: F(65535.0),
        11: F(0.95) * F(65535.0) / F(8.0), 12: F(0.95) * F(65535.0) / F(32.0), 13: F(6.0)}
MODE_BITS = {0: 10, 1: 7, 2: 11, 5: 9, 6: 8, 9: 6, 10: 10, 11: 11, 12: 12, 13: 16}


def unpack_to_uf16(v, bits):
    """bc6h.rs:199-211 with per-block bits."""
    v = np.asarray(v, np.int64)
    out = ((v * 2 + 1) << np.clip(15 - bits, 0, 15))
    out = np.where(v == (1 << bits) - 1, 0xFFFF, out)
    out = np.where(v == 0, 0, out)
    return np.where(bits >= 15, v, out)


def bit_at(v, pos):
    return (np.asarray(v, np.int64) >> pos) & 1


def reverse_bits(v, bits):
    """bc6h.rs:452-463."""
    v = np.asarray(v, np.int64)
    if bits == 2:
        return (v >> 1) + (v & 1) * 2
    vv = (v & 0x5555) * 2 + ((v >> 1) & 0x5555)
    return (vv >> 4) + ((vv >> 2) & 3) * 4 + (vv & 3) * 16


def pack(qep, mode):
    """bc6h_pack (bc6h.rs:465-791) for one mode over all blocks: (n, 4)."""
    n = qep.shape[0]
    q = lambda i: qep[:, i]  # noqa: E731
    packed = np.zeros((n, 4), np.int64)
    if mode <= 8:
        if mode == 0:
            mk = [31, 31, 31]
        elif mode == 1:
            mk = [63, 63, 63]
        elif mode in (2, 3, 4):
            mk = [31 if p == mode - 2 else 15 for p in range(3)]
        elif mode == 5:
            mk = [31, 31, 31]
        else:
            mk = [63 if p == mode - 6 else 31 for p in range(3)]
        d = {}
        for p in range(3):
            d[p] = q(p)
            d[4 + p] = (q(4 + p) - q(p)) & mk[p]
            d[8 + p] = (q(8 + p) - q(p)) & mk[p]
            d[12 + p] = (q(12 + p) - q(p)) & mk[p]
        pq = {i: np.zeros(n, np.int64) for i in range(10)}
        if mode == 0:
            pq[4] = d[4] + (d[9] & 15) * 64
            pq[5] = d[5] + (d[13] & 15) * 64
            pq[6] = d[6] + (d[10] & 15) * 64
            pq[4] += bit_at(d[13], 4) << 5
            pq[5] += bit_at(d[14], 0) << 5
            pq[6] += bit_at(d[14], 1) << 5
            pq[8] = d[8] + bit_at(d[14], 2) * 32
            pq[9] = d[12] + bit_at(d[14], 3) * 32
            packed[:, 0] = PREFIX[0] + (bit_at(d[9], 4) << 2) + (bit_at(d[10], 4) << 3) + (bit_at(d[14], 4) << 4)
            packed[:, 1] = (d[2] << 20) + (d[1] << 10) + d[0]
            packed[:, 2] = (pq[6] << 20) + (pq[5] << 10) + pq[4]
            packed[:, 3] = (pq[9] << 6) + pq[8]
        elif mode == 1:
            pq[0] = d[0] + (bit_at(d[14], 0) << 7) + (bit_at(d[14], 1) << 8) + (bit_at(d[10], 4) << 9)
            pq[1] = d[1] + (bit_at(d[10], 5) << 7) + (bit_at(d[14], 2) << 8) + (bit_at(d[9], 4) << 9)
            pq[2] = d[2] + (bit_at(d[14], 3) << 7) + (bit_at(d[14], 5) << 8) + (bit_at(d[14], 4) << 9)
            pq[4] = d[4] + (d[9] & 15) * 64
            pq[5] = d[5] + (d[13] & 15) * 64
            pq[6] = d[6] + (d[10] & 15) * 64
            packed[:, 0] = PREFIX[1] + (bit_at(d[9], 5) << 2) + (bit_at(d[13], 4) << 3) + (bit_at(d[13], 5) << 4)
            packed[:, 1] = (pq[2] << 20) + (pq[1] << 10) + pq[0]
            packed[:, 2] = (pq[6] << 20) + (pq[5] << 10) + pq[4]
            packed[:, 3] = (d[12] << 6) + d[8]
        else:
            if mode in (2, 3, 4):
                pq[0], pq[1], pq[2] = d[0] & 1023, d[1] & 1023, d[2] & 1023
            else:
                pq[0], pq[1], pq[2] = d[0].copy(), d[1].copy(), d[2].copy()
            pq[4] = d[4] + (d[9] & 15) * 64
            pq[5] = d[5] + (d[13] & 15) * 64
            pq[6] = d[6] + (d[10] & 15) * 64
            pq[8] = d[8].copy()
            pq[9] = d[12].copy()
            if mode == 2:
                pq[5] += bit_at(d[1], 10) << 4
                pq[6] += bit_at(d[2], 10) << 4
                pq[4] += bit_at(d[0], 10) << 5
                pq[5] += bit_at(d[14], 0) << 5
                pq[6] += bit_at(d[14], 1) << 5
                pq[8] += bit_at(d[14], 2) << 5
                pq[9] += bit_at(d[14], 3) << 5
            elif mode == 3:
                pq[4] += bit_at(d[0], 10) << 4
                pq[6] += bit_at(d[2], 10) << 4
                pq[8] += bit_at(d[14], 0) << 4
                pq[9] += bit_at(d[9], 4) << 4
                pq[4] += bit_at(d[13], 4) << 5
                pq[5] += bit_at(d[1], 10) << 5
                pq[6] += bit_at(d[14], 1) << 5
                pq[8] += bit_at(d[14], 2) << 5
                pq[9] += bit_at(d[14], 3) << 5
            elif mode == 4:
                pq[4] += bit_at(d[0], 10) << 4
                pq[5] += bit_at(d[1], 10) << 4
                pq[8] += bit_at(d[14], 1) << 4
                pq[9] += bit_at(d[14], 4) << 4
                pq[4] += bit_at(d[10], 4) << 5
                pq[5] += bit_at(d[14], 0) << 5
                pq[6] += bit_at(d[2], 10) << 5
                pq[8] += bit_at(d[14], 2) << 5
                pq[9] += bit_at(d[14], 3) << 5
            elif mode == 5:
                pq[0] += bit_at(d[10], 4) << 9
                pq[1] += bit_at(d[9], 4) << 9
                pq[2] += bit_at(d[14], 4) << 9
                pq[4] += bit_at(d[13], 4) << 5
                pq[5] += bit_at(d[14], 0) << 5
                pq[6] += bit_at(d[14], 1) << 5
                pq[8] += bit_at(d[14], 2) << 5
                pq[9] += bit_at(d[14], 3) << 5
            else:  # 6, 7, 8
                pq[0] += bit_at(d[10], 4) << 9
                pq[1] += bit_at(d[9], 4) << 9
                pq[2] += bit_at(d[14], 4) << 9
                if mode == 6:
                    pq[0] += bit_at(d[13], 4) << 8
                    pq[1] += bit_at(d[14], 2) << 8
                    pq[2] += bit_at(d[14], 3) << 8
                    pq[5] += bit_at(d[14], 0) << 5
                    pq[6] += bit_at(d[14], 1) << 5
                elif mode == 7:
                    pq[0] += bit_at(d[14], 0) << 8
                    pq[1] += bit_at(d[9], 5) << 8
                    pq[2] += bit_at(d[13], 5) << 8
                    pq[4] += bit_at(d[13], 4) << 5
                    pq[6] += bit_at(d[14], 1) << 5
                    pq[8] += bit_at(d[14], 2) << 5
                    pq[9] += bit_at(d[14], 3) << 5
                else:
                    pq[0] += bit_at(d[14], 1) << 8
                    pq[1] += bit_at(d[10], 5) << 8
                    pq[2] += bit_at(d[14], 5) << 8
                    pq[4] += bit_at(d[13], 4) << 5
                    pq[5] += bit_at(d[14], 0) << 5
                    pq[8] += bit_at(d[14], 2) << 5
                    pq[9] += bit_at(d[14], 3) << 5
            packed[:, 0] = PREFIX[mode]
            packed[:, 1] = (pq[2] << 20) + (pq[1] << 10) + pq[0]
            packed[:, 2] = (pq[6] << 20) + (pq[5] << 10) + pq[4]
            packed[:, 3] = (pq[9] << 6) + pq[8]
    elif mode == 9:
        p0 = q(0) + (bit_at(q(13), 4) << 6) + (bit_at(q(14), 0) << 7) + (bit_at(q(14), 1) << 8) + (bit_at(q(10), 4) << 9)
        p1 = q(1) + (bit_at(q(9), 5) << 6) + (bit_at(q(10), 5) << 7) + (bit_at(q(14), 2) << 8) + (bit_at(q(9), 4) << 9)
        p2 = q(2) + (bit_at(q(13), 5) << 6) + (bit_at(q(14), 3) << 7) + (bit_at(q(14), 5) << 8) + (bit_at(q(14), 4) << 9)
        p4 = q(4) + (q(9) & 15) * 64
        p5 = q(5) + (q(13) & 15) * 64
        p6 = q(6) + (q(10) & 15) * 64
        packed[:, 0] = PREFIX[9]
        packed[:, 1] = (p2 << 20) + (p1 << 10) + p0
        packed[:, 2] = (p6 << 20) + (p5 << 10) + p4
        packed[:, 3] = (q(12) << 6) + q(8)
    elif mode == 10:
        packed[:, 0] = PREFIX[10]
        packed[:, 1] = (q(2) << 20) + (q(1) << 10) + q(0)
        packed[:, 2] = (q(6) << 20) + (q(5) << 10) + q(4)
    else:  # 11, 12, 13
        m = {11: 511, 12: 255, 13: 15}[mode]
        d = {p: q(p) for p in range(3)}
        for p in range(3):
            d[4 + p] = (q(4 + p) - q(p)) & m
        hi = {}
        for p in range(3):
            if mode == 11:
                hi[p] = (d[p] >> 10) * 512
            elif mode == 12:
                hi[p] = reverse_bits(d[p] >> 10, 2) * 256
            else:
                hi[p] = reverse_bits(d[p] >> 10, 6) * 16
        packed[:, 0] = PREFIX[mode]
        packed[:, 1] = ((d[2] & 1023) << 20) + ((d[1] & 1023) << 10) + (d[0] & 1023)
        packed[:, 2] = ((d[6] + hi[2]) << 20) + ((d[5] + hi[1]) << 10) + (d[4] + hi[0])
    return packed & U32


def pack_per_block(qep, modes):
    out = np.zeros((qep.shape[0], 4), np.int64)
    for m in np.unique(modes):
        sel = modes == m
        out[sel] = pack(qep[sel], int(m))
    return out


class Encoder:
    """State of compress_bc6h_core (bc6h.rs:793-860) for n blocks."""

    def __init__(self, block, settings):
        self.block = np.array(block, F)
        s = [int(x) for x in settings]
        self.slow, self.fast, self.ref1, self.ref2, self.k = s
        n = self.block.shape[0]
        self.n = n
        self.best_err = np.full(n, INF, F)
        self.data = np.zeros((n, 4), np.int64)
        self.mode = np.zeros(n, np.int64)
        self.epb = np.zeros(n, np.int64)
        self.qb = np.zeros((n, 8), np.int64)
        self._list = None
        # bc6h_setup (bc6h.rs:793-819)
        lo = [np.full(n, 65535.0, F) for _ in range(3)]
        hi = [np.zeros(n, F) for _ in range(3)]
        for p in range(3):
            for k in range(16):
                v = (self.block[:, p * 16 + k] / F(31.0)) * F(64.0)
                self.block[:, p * 16 + k] = v
                lo[p] = np.fmin(lo[p], v)
                hi[p] = np.fmax(hi[p], v)
        self.bounds = lo + hi
        self.max_span = np.zeros(n, F)
        self.max_span_idx = np.zeros(n, np.int64)
        for p in range(3):
            span = hi[p] - lo[p]
            up = span > self.max_span
            self.max_span_idx = np.where(up, p, self.max_span_idx)
            self.max_span = np.where(up, span, self.max_span)

    def qbounds(self, sel, spans, epb):
        """compute_qbounds_core + ep_quant_bc6h_8 (bc6h.rs:166-189) on the blocks in `sel`."""
        levels = np.int64(1) << epb
        for p in range(3):
            middle = (self.bounds[p] + self.bounds[3 + p]) / F(2.0)
            lo = middle - spans[p] / F(2.0)
            hi = middle + spans[p] / F(2.0)
            for i, b in ((p, lo), (4 + p, hi)):
                v = nr.as_int(b / F(65535.0) * (levels - 1).astype(F) + F(0.5))
                self.qb[:, i] = np.where(sel, np.clip(v, 0, levels - 1), self.qb[:, i])
        for i in (3, 7):  # the padding entries of the 8 quantised bounds
            self.qb[:, i] = np.where(sel, 0, self.qb[:, i])

    def test_mode(self, mode, enc, margin):
        """bc6h_test_mode (bc6h.rs:414-446): returns the blocks that passed
        (their state is set; the others keep theirs)."""
        span = SPAN[mode]
        ok = ~(self.max_span * F(margin) > span)
        epb = MODE_BITS[mode]
        self.epb = np.where(ok, epb, self.epb)
        n = self.n
        if mode >= 10 or mode <= 1 or mode in (5, 9):
            self.mode = np.where(ok, mode, self.mode)
            self.qbounds(ok, [np.full(n, span, F)] * 3, np.full(n, epb, np.int64))
        else:
            self.mode = np.where(ok, mode + self.max_span_idx, self.mode)
            spans = [np.where(self.max_span_idx == p, span * F(2.0), span).astype(F) for p in range(3)]
            self.qbounds(ok, spans, np.full(n, epb, np.int64))
        if enc:
            if mode >= 10:
                self.enc_1p(ok)
            else:
                self.enc_2p(ok)
        return ok

    def quant_dequant(self, ep, pairs):
        """ep_quant_dequant_bc6h (bc6h.rs:213-239)."""
        levels = np.int64(1) << self.epb
        qep = np.zeros((self.n, 24), np.int64)
        ep = ep.copy()
        for i in range(8 * pairs):
            v = nr.as_int(ep[:, i] / F(65535.0) * (levels - 1).astype(F) + F(0.5))
            qep[:, i] = np.clip(v, 0, levels - 1)
        for i in range(2 * pairs):
            for p in range(3):
                qep[:, i * 4 + p] = np.clip(qep[:, i * 4 + p], self.qb[:, p], self.qb[:, 4 + p])
        for i in range(8 * pairs):
            ep[:, i] = unpack_to_uf16(qep[:, i], self.epb).astype(F)
        return qep, ep

    def part_list(self):
        """The 32 split bounds and the ascending top-k list (bc6h.rs:288-302);
        the keys are unique, so partial_sort_list's first k entries are the k
        smallest. The bounds depend only on the block, so one list serves every
        two-region encode."""
        if self._list is None:
            keys = np.zeros((self.n, 32), np.int64)
            for part in range(32):
                mask = np.full(self.n, b7.pattern_mask(np.array([part]), 0)[0], np.int64)
                b12 = nr.block_pca_bound_split(self.block, mask, 3)
                keys[:, part] = part + nr.as_int(b12) * 64
            self._list = np.sort(keys, axis=1)[:, :self.k] & 31
        return self._list

    def enc_2p(self, sel):
        """bc6h_enc_2p + bc6h_enc_2p_list (bc6h.rs:288-388) for the blocks in `sel`."""
        if self.k == 0:
            return
        lst = self.part_list()
        n = self.n
        best_qep = np.zeros((n, 24), np.int64)
        best_q = np.zeros((n, 2), np.int64)
        best_part = np.full(n, -1, np.int64)
        best = np.full(n, INF, F)
        for c in range(self.k):
            part = lst[:, c]
            ep = np.zeros((n, 24), F)
            for j in range(2):
                ep[:, 8 * j:8 * j + 8] = nr.block_segment_core(self.block, b7.pattern_mask(part, j), 3)
            qep, ep = self.quant_dequant(ep, 2)
            qblock, err = nr.block_quant(self.block, 3, ep, b7.PATTERN[part], 3)
            up = err < best
            best_qep[:, :16] = np.where(up[:, None], qep[:, :16], best_qep[:, :16])
            best_q = np.where(up[:, None], qblock.astype(np.int64), best_q)
            best_part = np.where(up, part, best_part)
            best = np.where(up, err, best)
        found = best_part >= 0
        bp = np.where(found, best_part, 0)
        for _ in range(self.ref2):
            ep = np.zeros((n, 24), F)
            for j in range(2):
                ep[:, 8 * j:8 * j + 8] = nr.opt_endpoints(ep[:, 8 * j:8 * j + 8], self.block, 3, best_q,
                                                          b7.pattern_mask(bp, j), 3)
            qep, ep = self.quant_dequant(ep, 2)
            qblock, err = nr.block_quant(self.block, 3, ep, b7.PATTERN[bp], 3)
            up = (err < best) & found
            best_qep[:, :16] = np.where(up[:, None], qep[:, :16], best_qep[:, :16])
            best_q = np.where(up[:, None], qblock.astype(np.int64), best_q)
            best = np.where(up, err, best)
        win = sel & found & (best < self.best_err)
        if win.any():
            coded = self.code_2p(best_qep, best_q, bp)
            self.data = np.where(win[:, None], coded, self.data)
            self.best_err = np.where(win, best, self.best_err)

    def enc_1p(self, sel):
        """bc6h_enc_1p (bc6h.rs:390-412) for the blocks in `sel`."""
        n = self.n
        ep = np.zeros((n, 24), F)
        ep[:, :8] = nr.block_segment_core(self.block, np.full(n, 0xFFFFFFFF, np.int64), 3)
        qep, ep = self.quant_dequant(ep, 1)
        zero = np.zeros(n, np.int64)
        qblock, err = nr.block_quant(self.block, 4, ep, zero, 3)
        full = np.full(n, 0xFFFFFFFF, np.int64)
        for _ in range(self.ref1):
            ep[:, :8] = nr.opt_endpoints(ep[:, :8], self.block, 4, qblock, full, 3)
            qep, ep = self.quant_dequant(ep, 1)
            qblock, err = nr.block_quant(self.block, 4, ep, zero, 3)
        win = sel & (err < self.best_err)
        if win.any():
            coded = self.code_1p(qep, qblock.astype(np.int64))
            self.data = np.where(win[:, None], coded, self.data)
            self.best_err = np.where(win, err, self.best_err)

    def code_2p(self, qep, qblock, part):
        """bc6h_code_2p (bc6h.rs:241-266)."""
        qep, qblock = qep.copy(), qblock.copy()
        flips = b7.apply_swap_mode01237(qep, qblock, 1, part)
        packed = pack_per_block(qep, self.mode)
        data = np.zeros((self.n, 5), np.int64)
        pos = b7.put_bits(data, 0, 5, packed[:, 0])
        pos = b7.put_bits(data, pos, 30, packed[:, 1])
        pos = b7.put_bits(data, pos, 30, packed[:, 2])
        pos = b7.put_bits(data, pos, 12, packed[:, 3])
        pos = b7.put_bits(data, pos, 5, part)
        pos = b7.code_qblock(data, pos, qblock, 3, flips)
        sk = b7.skips(part)
        b7.data_shl_1bit_from(data, 128 + 1 - (15 - sk[:, 1]) * 3)
        return data[:, :4]

    def code_1p(self, qep, qblock):
        """bc6h_code_1p (bc6h.rs:268-286)."""
        qep, qblock = qep.copy(), qblock.copy()
        b7.apply_swap_mode456(qep, 4, qblock, 4)
        packed = pack_per_block(qep, self.mode)
        data = np.zeros((self.n, 5), np.int64)
        pos = b7.put_bits(data, 0, 5, packed[:, 0])
        pos = b7.put_bits(data, pos, 30, packed[:, 1])
        pos = b7.put_bits(data, pos, 30, packed[:, 2])
        pos = b7.code_qblock(data, pos, qblock, 4, np.zeros(self.n, np.int64))
        return data[:, :4]

    def encode(self):
        """compress_bc6h_core (bc6h.rs:821-860): (n, 4) uint32 words."""
        if self.slow:
            for m in (0, 1, 2, 5, 6, 9, 10, 11, 12, 13):
                self.test_mode(m, True, 0.0)
        else:
            if self.k > 0:
                self.test_mode(9, False, 0.0)
                if self.fast:
                    self.test_mode(1, False, 1.0)
                self.test_mode(6, False, 1.0 / 1.2)
                self.test_mode(5, False, 1.0 / 1.2)
                self.test_mode(0, False, 1.0 / 1.2)
                self.test_mode(2, False, 1.0)
                self.enc_2p(np.ones(self.n, bool))
                if not self.fast:
                    self.test_mode(1, True, 0.0)
            self.test_mode(10, False, 0.0)
            self.test_mode(11, False, 1.0)
            self.test_mode(12, False, 1.0)
            self.test_mode(13, False, 1.0)
            self.enc_1p(np.ones(self.n, bool))
        return (self.data & U32).astype(np.uint32)


def compress_bc6h(rgba16, settings):
    """compress_bc6h_16bit (src/encode.rs:590-620) of an (h, w, 4) array of f16
    bit patterns (uint16) -> the packed little-endian 16-byte blocks."""
    h, w = rgba16.shape[:2]
    t = np.asarray(rgba16, np.uint16).reshape(h // 4, 4, w // 4, 4, 4).transpose(0, 2, 4, 1, 3)
    blocks = np.ascontiguousarray(t.reshape(-1, 64)).astype(F)
    blocks[:, 48:64] = 0.0  # load_block_interleaved_16bit leaves alpha 0
    words = Encoder(blocks, settings).encode()
    return np.ascontiguousarray(words.astype("<u4")).view(np.uint8).reshape(-1)
