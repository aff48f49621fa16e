"""Pure-Python restatement of the GPU Zstd entropy stage (test checker only):
one frame per window from its ZSTD_Sequence records, following RFC 8878 --
single-segment frame header, one block, literals raw, RLE or Huffman-coded
(whichever is smallest), sequences with repeat-offset codes and, per field
(LL, OF, ML), an RLE, FSE-compressed or predefined table chosen by the GPU's
integer cost estimate -- or a raw block when the compressed block would not be
smaller than the window.  The tests compare the GPU frames
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


# ------------------------------------------------------------------ literals

HUF_MAX_BITS = 11


def _huffman_lengths(counts):
    """Code lengths of a Huffman code over the present symbols (two queues;
    leaves sorted by (count, symbol); on equal counts the leaf is taken
    first), limited to HUF_MAX_BITS by moving pairs of leaves up the tree
    while keeping the code complete."""
    leaves = sorted((c, s) for s, c in enumerate(counts) if c)
    n = len(leaves)
    cnt = [c for c, _ in leaves] + [0] * (n - 1)
    parent = [0] * (2 * n - 1)
    li, ii, nxt = 0, n, n

    def pop():
        nonlocal li, ii
        if li < n and (ii >= nxt or cnt[li] <= cnt[ii]):
            li += 1
            return li - 1
        ii += 1
        return ii - 1

    while nxt < 2 * n - 1:
        a = pop()
        b = pop()
        cnt[nxt] = cnt[a] + cnt[b]
        parent[a] = parent[b] = nxt
        nxt += 1
    depth = [0] * (2 * n - 1)
    for k in range(2 * n - 3, -1, -1):
        depth[k] = depth[parent[k]] + 1
    bl = [0] * 64
    for k in range(n):
        bl[depth[k]] += 1
    maxlen = max(depth[:n])
    for i in range(maxlen, HUF_MAX_BITS, -1):
        while bl[i] > 0:
            j = i - 2
            while bl[j] == 0:
                j -= 1
            bl[i] -= 2
            bl[i - 1] += 1
            bl[j + 1] += 2
            bl[j] -= 1
    # longest codes to the least frequent symbols
    lens = [0] * 256
    k = 0
    for length in range(HUF_MAX_BITS, 0, -1):
        for _ in range(bl[length]):
            lens[leaves[k][1]] = length
            k += 1
    return lens


def _canonical_codes(lens):
    maxb = max(lens)
    bl = [0] * (maxb + 2)
    for l in lens:
        if l:
            bl[l] += 1
    start = [0] * (maxb + 2)
    for l in range(maxb - 1, 0, -1):
        start[l] = (start[l + 1] + bl[l + 1]) >> 1
    codes = [0] * 256
    for s in range(256):
        if lens[s]:
            codes[s] = start[lens[s]]
            start[lens[s]] += 1
    return codes


def _ncount_bits(norm, al, bits):
    """FSE table description (RFC 8878 4.1.1) of `norm` (no -1 entries)."""
    bits.add(al - 5, 4)
    remaining, threshold, nb = (1 << al) + 1, 1 << al, al + 1
    last = max(s for s, c in enumerate(norm) if c)
    s = 0
    while s <= last:
        v = norm[s] + 1
        mx = (2 * threshold - 1) - remaining
        if v < mx:
            bits.add(v, nb - 1)
        elif v < threshold:
            bits.add(v, nb)
        else:
            bits.add(v + mx, nb)
        remaining -= norm[s]
        while remaining < threshold:
            nb -= 1
            threshold >>= 1
        if norm[s] == 0:
            z = 0
            while s + 1 + z < last and norm[s + 1 + z] == 0:
                z += 1
            s += z
            while z >= 3:
                bits.add(3, 2)
                z -= 3
            bits.add(z, 2)
        s += 1


def _fse_dec_table(norm, al):
    size = 1 << al
    mask, step, high = size - 1, (size >> 1) + (size >> 3) + 3, size - 1
    sym = [0] * size
    nxt = list(norm)
    pos = 0
    for s, c in enumerate(norm):
        for _ in range(c):
            sym[pos] = s
            pos = (pos + step) & mask
            while pos > high:
                pos = (pos + step) & mask
    nbits, base = [0] * size, [0] * size
    for u in range(size):
        x = nxt[sym[u]]
        nxt[sym[u]] += 1
        nbits[u] = al - (x.bit_length() - 1)
        base[u] = (x << nbits[u]) - size
    return sym, nbits, base


def _fse_weights(weights):
    """FSE-compressed Huffman weights (accuracy 6, two interleaved states), or
    None when that is not possible or larger than 127 bytes."""
    al, size = 6, 64
    n = len(weights)
    cw = [0] * 12
    for w in weights:
        cw[w] += 1
    if sum(1 for c in cw if c) < 2:
        return None
    norm = [0 if c == 0 else max(1, c * size // n) for c in cw]
    big = max(range(12), key=lambda s: (norm[s], -s))
    norm[big] += size - sum(norm)
    if norm[big] <= 0:
        return None
    sym, nbits, base = _fse_dec_table(norm, al)
    enc = {}
    for u in range(size):
        for v in range(base[u], base[u] + (1 << nbits[u])):
            enc[(sym[u], v)] = u
    bits = _Bits()
    _ncount_bits(norm, al, bits)
    desc = bits.v.to_bytes((bits.n + 7) // 8, "little")
    st = [0] * n
    st[n - 1] = next(u for u in range(size) if sym[u] == weights[n - 1])
    st[n - 2] = next(u for u in range(size) if sym[u] == weights[n - 2] and nbits[u] >= 1)
    for i in range(n - 3, -1, -1):
        st[i] = enc[(weights[i], st[i + 2])]
    b2 = _Bits()
    for i in range(n - 3, -1, -1):
        b2.add(st[i + 2] - base[st[i]], nbits[st[i]])
    b2.add(st[1], al)
    b2.add(st[0], al)
    out = desc + b2.close()
    return out if len(out) <= 127 else None


def _huf_stream(data, lens, codes):
    bits = _Bits()
    for x in reversed(data):
        bits.add(codes[x], lens[x])
    return bits.close()


def _raw_lit_header(btype, n):
    if n < 32:
        return bytes([btype | (n << 3)])
    if n < 4096:
        return bytes([btype | 4 | ((n << 4) & 0xF0), n >> 4])
    return bytes([btype | 12 | ((n << 4) & 0xF0), (n >> 4) & 0xFF, n >> 12])


def literals_section(lits):
    """Smallest of: raw, RLE (one distinct byte), Huffman-compressed (1 stream
    below 1024 literals, else 4 streams)."""
    lits = bytes(lits)
    nl = len(lits)
    raw = _raw_lit_header(0, nl) + lits
    if nl == 0:
        return raw
    counts = [0] * 256
    for x in lits:
        counts[x] += 1
    if sum(1 for c in counts if c) == 1:
        return _raw_lit_header(1, nl) + lits[:1]
    lens = _huffman_lengths(counts)
    maxb = max(lens)
    last = max(s for s in range(256) if counts[s])
    weights = [(maxb + 1 - lens[s]) if lens[s] else 0 for s in range(last)]
    if len(weights) <= 128:
        packed = bytes([127 + len(weights)])
        ws = weights + [0]
        packed += bytes((ws[i] << 4) | ws[i + 1] for i in range(0, len(weights), 2))
        tree = packed
    else:
        f = _fse_weights(weights)
        if f is None:
            return raw
        tree = bytes([len(f)]) + f
    codes = _canonical_codes(lens)
    if nl < 1024:
        streams = [_huf_stream(lits, lens, codes)]
        body = tree + streams[0]
        if len(body) >= 1024:
            return raw
        hdr = (2 | (0 << 2) | (nl << 4) | (len(body) << 14)).to_bytes(3, "little")
    else:
        seg = (nl + 3) // 4
        parts = [lits[k * seg:(k + 1) * seg] for k in range(3)] + [lits[3 * seg:]]
        streams = [_huf_stream(p, lens, codes) for p in parts]
        if any(len(s) > 65535 for s in streams[:3]):
            return raw
        body = tree + b"".join(len(s).to_bytes(2, "little") for s in streams[:3]) + b"".join(streams)
        m = max(nl, len(body))
        if m < 16384:
            hdr = (2 | (2 << 2) | (nl << 4) | (len(body) << 18)).to_bytes(4, "little")
        else:
            hdr = (2 | (3 << 2) | (nl << 4) | (len(body) << 22)).to_bytes(5, "little")
    out = hdr + body
    return out if len(out) < len(raw) else raw


def _lg256(x):
    """log2(x) * 256, piecewise linear between powers of two (integer)."""
    h = x.bit_length() - 1
    return 256 * h + ((x << 8) >> h) - 256


def _seq_table(hist, pre_norm, pre_log, amax):
    """The table of one sequence field (RFC 8878 3.1.1.3.2.1): ("rle", code),
    ("fse", norm, accuracy, description) or ("pre",), by the same integer cost
    estimate as the GPU: k * (A * 256 - lg256(n)) per code used k times with
    normalised count n, plus 2048 per description byte."""
    ns = sum(hist)
    used = [c for c, k in enumerate(hist) if k]
    if len(used) == 1:
        return ("rle", used[0])
    last = used[-1]
    pre_ok = all(c < len(pre_norm) and pre_norm[c] != 0 for c in used)
    cost_pre = sum(hist[c] * (256 * pre_log - _lg256(1 if pre_norm[c] < 0 else pre_norm[c])) for c in used) \
        if pre_ok else None
    al = max(5, min(amax, max((ns - 1).bit_length() - 2, 0)))
    while (1 << al) < 2 * len(used) and al < amax:
        al += 1
    size = 1 << al
    norm = [0] * (last + 1)
    for c in used:
        norm[c] = max(1, (hist[c] * size + ns // 2) // ns)
    top = max(used, key=lambda c: (hist[c], -c))
    d = size - sum(norm)
    if d > 0:
        norm[top] += d
    while d < 0:
        big = max(range(last + 1), key=lambda c: (norm[c], -c))
        norm[big] -= 1
        d += 1
    bits = _Bits()
    _ncount_bits(norm, al, bits)
    desc = bits.v.to_bytes((bits.n + 7) // 8, "little")
    cost_fse = 2048 * len(desc) + sum(hist[c] * (256 * al - _lg256(norm[c])) for c in used)
    if len(desc) <= 128 and (cost_pre is None or cost_fse < cost_pre):
        return ("fse", norm, al, desc)
    return ("pre",)


MODE_USES = {"rle": 0, "fse": 0, "pre": 0}  # tables chosen so far (for the tests' coverage checks)


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
    lsec = literals_section(lits)
    ns = len(seqs)
    sh = bytes([ns]) if ns < 128 else bytes([(ns >> 8) + 0x80, ns & 0xFF])
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
    lcs = [_code(LL_BASE, ll) for _, ll, _ in seqs]
    mcs = [_code(ML_BASE, ml) for _, _, ml in seqs]
    ocs = [v.bit_length() - 1 for v in ovs]
    # tables: LL, OF, ML (the order of the modes byte and of the descriptions)
    modes, descs, enc, logs = 0, b"", {}, {}
    for key, codes, ncodes, pre, pre_log, amax, shift, pre_enc in (
            ("ll", lcs, 36, LL_NORM, LL_LOG, 9, 6, ENC_LL), ("of", ocs, 32, OF_NORM, OF_LOG, 8, 4, ENC_OF),
            ("ml", mcs, 53, ML_NORM, ML_LOG, 9, 2, ENC_ML)):
        hist = [0] * ncodes
        for c in codes:
            hist[c] += 1
        t = _seq_table(hist, pre, pre_log, amax)
        MODE_USES[t[0]] += 1
        if t[0] == "rle":
            modes |= 1 << shift
            descs += bytes([t[1]])
            enc[key], logs[key] = None, 0
        elif t[0] == "fse":
            modes |= 2 << shift
            descs += t[3]
            enc[key], logs[key] = _fse(t[1], t[2]), t[2]
        else:
            enc[key], logs[key] = pre_enc, pre_log
    sh += bytes([modes]) + descs
    bits = _Bits()
    st = {"ll": 0, "ml": 0, "of": 0}
    for i in range(ns - 1, -1, -1):
        _, ll, ml = seqs[i]
        v = ovs[i]
        lc, mc, oc = lcs[i], mcs[i], ocs[i]
        code = {"ll": lc, "ml": mc, "of": oc}
        if i == ns - 1:  # any state of the code, no bits
            for k in ("ll", "ml", "of"):
                st[k] = enc[k][(code[k], 0)][0] if enc[k] is not None else 0
        else:
            for k in ("of", "ml", "ll"):
                if enc[k] is None:  # RLE_Mode: no state, no bits
                    continue
                u, nb, base = enc[k][(code[k], st[k])]
                bits.add(st[k] - base, nb)
                st[k] = u
        bits.add(ll - LL_BASE[lc], LL_BITS[lc])
        bits.add(ml - ML_BASE[mc], ML_BITS[mc])
        bits.add(v - (1 << oc), oc)
    bits.add(st["ml"], logs["ml"])
    bits.add(st["of"], logs["of"])
    bits.add(st["ll"], logs["ll"])
    content = lsec + sh + bits.close()
    if len(content) >= w:
        return raw
    return fh + _block_header(2, len(content)) + content
