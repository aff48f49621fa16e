"""Pure-Python restatement of the GPU Zstd entropy stage (test checker only):
one frame per window from its ZSTD_Sequence records, following RFC 8878 --
single-segment frame header, one block, Raw_Literals_Block, sequences in
Predefined_Mode with repeat-offset codes -- or a raw block when the compressed
block would not be smaller than the window.  The tests compare the GPU frames
with these byte for byte and decode both with stock libzstd."""

LL_NORM = [4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1,
           -1, -1, -1, -1]
ML_NORM = [1, 4, 3, 2, 2, 2, 2, 2, 2] + [1] * 37 + [-1] * 7
OF_NORM = [1, 1, 1, 1, 1, 1, 2, 2, 2] + [1] * 15 + [-1] * 5
LL_LOG, ML_LOG, OF_LOG = 6, 6, 5

LL_BASE = list(range(16)) + [16, 18, 20, 22, 24, 28, 32, 40, 48, 64] + [1 << k for k in range(7, 17)]
LL_BITS = [0] * 16 + [1, 1, 1, 1, 2, 2, 3, 3, 4, 6] + list(range(7, 17))
ML_BASE = list(range(3, 35)) + [35, 37, 39, 41, 43, 47, 51, 59, 67, 83, 99, 131] + [(1 << k) + 3 for k in range(8, 17)]
ML_BITS = [0] * 32 + [1, 1, 1, 1, 2, 2, 3, 3, 4, 4, 5, 7] + list(range(8, 17))


def _fse(norm, al):
    """Decoder spread + per-state nbBits/baseline (RFC 8878 4.1.1), as an
    encoder map (symbol, next decoder state) -> (state, nbBits, baseline)."""
    size = 1 << al
    mask, step, high = size - 1, (size >> 1) + (size >> 3) + 3, size - 1
    sym = [0] * size
    nxt = {}
    for s, c in enumerate(norm):
        if c == -1:
            sym[high] = s
            high -= 1
            nxt[s] = 1
        else:
            nxt[s] = c
    pos = 0
    for s, c in enumerate(norm):
        for _ in range(max(c, 0)):
            sym[pos] = s
            pos = (pos + step) & mask
            while pos > high:
                pos = (pos + step) & mask
    enc = {}
    for u in range(size):
        x = nxt[sym[u]]
        nxt[sym[u]] += 1
        nb = al - (x.bit_length() - 1)
        base = (x << nb) - size
        for v in range(base, base + (1 << nb)):
            enc[(sym[u], v)] = (u, nb, base)
    return enc


ENC_LL, ENC_ML, ENC_OF = _fse(LL_NORM, LL_LOG), _fse(ML_NORM, ML_LOG), _fse(OF_NORM, OF_LOG)


def _code(bases, v):
    return max(i for i, b in enumerate(bases) if b <= v)


class _Bits:
    def __init__(self):
        self.v = 0
        self.n = 0

    def add(self, val, nb):
        self.v |= val << self.n
        self.n += nb

    def close(self):
        self.add(1, 1)
        return self.v.to_bytes((self.n + 7) // 8, "little")


def _frame_header(w):
    if w < 256:
        return b"\x28\xb5\x2f\xfd" + bytes([0x20, w])
    return b"\x28\xb5\x2f\xfd" + bytes([0x60]) + (w - 256).to_bytes(2, "little")


def _block_header(btype, size):
    return (1 | (btype << 1) | (size << 3)).to_bytes(3, "little")


def encode_frame(win, seqs):
    """win: bytes of one window; seqs: iterable of (offset, litLength, matchLength)."""
    win = bytes(win)
    w = len(win)
    seqs = [(int(o), int(ll), int(ml)) for o, ll, ml in seqs]
    fh = _frame_header(w)
    raw = fh + _block_header(0, w) + win
    if not seqs:
        return raw
    lits, pos = bytearray(), 0
    for o, ll, ml in seqs:
        lits += win[pos:pos + ll]
        pos += ll + ml
    lits += win[pos:]
    nl = len(lits)
    if nl < 32:
        lh = bytes([nl << 3])
    elif nl < 4096:
        lh = bytes([((nl << 4) & 0xF0) | 4, nl >> 4])
    else:
        lh = bytes([((nl << 4) & 0xF0) | 12, (nl >> 4) & 0xFF, nl >> 12])
    ns = len(seqs)
    sh = bytes([ns]) if ns < 128 else bytes([(ns >> 8) + 0x80, ns & 0xFF])
    sh += b"\x00"
    # repeat codes with the decoder's history
    r1, r2, r3 = 1, 4, 8
    ovs = []
    for o, ll, _ in seqs:
        if ll:
            v = 1 if o == r1 else 2 if o == r2 else 3 if o == r3 else o + 3
        else:
            v = 1 if o == r2 else 2 if o == r3 else 3 if o == r1 - 1 else o + 3
        if v > 3:
            r1, r2, r3 = o, r1, r2
        else:
            idx = v - 1 + (1 if ll == 0 else 0)
            if idx == 1:
                r1, r2 = o, r1
            elif idx >= 2:
                r1, r2, r3 = o, r1, r2
        ovs.append(v)
    bits = _Bits()
    dll = dml = dof = 0
    for i in range(ns - 1, -1, -1):
        _, ll, ml = seqs[i]
        v = ovs[i]
        lc, mc, oc = _code(LL_BASE, ll), _code(ML_BASE, ml), v.bit_length() - 1
        if i == ns - 1:
            dll, dml, dof = ENC_LL[(lc, 0)][0], ENC_ML[(mc, 0)][0], ENC_OF[(oc, 0)][0]
        else:
            for enc, cur, code in ((ENC_OF, "of", oc), (ENC_ML, "ml", mc), (ENC_LL, "ll", lc)):
                d = {"of": dof, "ml": dml, "ll": dll}[cur]
                u, nb, base = enc[(code, d)]
                bits.add(d - base, nb)
                if cur == "of":
                    dof = u
                elif cur == "ml":
                    dml = u
                else:
                    dll = u
        bits.add(ll - LL_BASE[lc], LL_BITS[lc])
        bits.add(ml - ML_BASE[mc], ML_BITS[mc])
        bits.add(v - (1 << oc), oc)
    bits.add(dml, ML_LOG)
    bits.add(dof, OF_LOG)
    bits.add(dll, LL_LOG)
    content = lh + bytes(lits) + sh + bits.close()
    if len(content) >= w:
        return raw
    return fh + _block_header(2, len(content)) + content
