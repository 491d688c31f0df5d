"""CPU restatement of the learned planner's device parts -- TEST INFRASTRUCTURE ONLY.

Used by tests (and nothing on the product path) to check the CUDA kernels:
  * sketch(keys, valid, n): the 280 features of nfc_sketch (HyperLogLog-256 registers
    from a splitmix64 hash of each valid key among the first 65,536 rows, plus 24 run /
    range statistics), in float64 arithmetic cast to float32;
  * bf16(x): round-to-nearest-even of float32 to bfloat16 (kept as float32 values);
  * mlp_forward / mlp_backward: the 280-128-128-5 ReLU network with bf16 weight
    matrices, float32 biases, in float64 -- the reference for the CUDA forward and
    backward passes (fp32 accumulation there);
  * mlp_loss: squared error on out[0] plus cross-entropy on out[1:5].

The reference project has no learned planner; its fixed rule is pinned separately
against the reference's own plan_groupby decisions (tests/golden/plan_fixed.json).
"""

import numpy as np

IN, H, OUT = 280, 128, 5
SKETCH_ROWS = 65536
REGS = 256
NPARAMS = IN * H + H + H * H + H + H * OUT + OUT

_M64 = (1 << 64) - 1


def offsets():
    w1 = 0
    b1 = w1 + IN * H
    w2 = b1 + H
    b2 = w2 + H * H
    w3 = b2 + H
    b3 = w3 + H * OUT
    return {"W1": (w1, (IN, H)), "b1": (b1, (H,)), "W2": (w2, (H, H)), "b2": (b2, (H,)),
            "W3": (w3, (H, OUT)), "b3": (b3, (OUT,))}


def unpack(params):
    p = np.asarray(params, dtype=np.float32)
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in offsets().items()}


def pack(d):
    out = np.zeros(NPARAMS, dtype=np.float32)
    for k, (o, s) in offsets().items():
        out[o:o + int(np.prod(s))] = np.asarray(d[k], dtype=np.float32).ravel()
    return out


def bf16(x):
    """float32 -> bfloat16 (round to nearest, ties to even), returned as float32."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    u = ((u + r) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def init_params(seed=0):
    """He-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, fan_in, fan_out in (("W1", IN, H), ("W2", H, H), ("W3", H, OUT)):
        lim = np.sqrt(6.0 / fan_in)
        d[name] = rng.uniform(-lim, lim, (fan_in, fan_out)).astype(np.float32)
    for name, n in (("b1", H), ("b2", H), ("b3", OUT)):
        d[name] = np.zeros(n, dtype=np.float32)
    return pack(d)


def mlp_forward(x, params, mu=None, sd=None):
    """Returns (xn, h1, h2, out) in float64, with bf16-rounded weight matrices."""
    p = unpack(params)
    x = np.asarray(x, dtype=np.float64)
    xn = x if mu is None else (x - np.asarray(mu, np.float64)) / np.asarray(sd, np.float64)
    w1, w2, w3 = (bf16(p[k]).astype(np.float64) for k in ("W1", "W2", "W3"))
    h1 = np.maximum(xn @ w1 + p["b1"], 0.0)
    h2 = np.maximum(h1 @ w2 + p["b2"], 0.0)
    out = h2 @ w3 + p["b3"]
    return xn, h1, h2, out


def mlp_loss(out, y, label, card_w, cls_w, weight=None):
    """Mean loss and d(mean loss)/d(out); weight scales each row's class term."""
    out = np.asarray(out, np.float64)
    b = out.shape[0]
    wcls = cls_w * (np.ones(b) if weight is None else np.asarray(weight, np.float64))
    e = out[:, 0] - y
    loss = card_w * e * e
    d = np.zeros_like(out)
    d[:, 0] = 2.0 * card_w * e / b
    lg = out[:, 1:]
    mx = lg.max(axis=1, keepdims=True)
    ex = np.exp(lg - mx)
    se = ex.sum(axis=1, keepdims=True)
    prob = ex / se
    has = label >= 0
    onehot = np.zeros_like(prob)
    onehot[np.arange(b)[has], label[has]] = 1.0
    d[:, 1:] = np.where(has[:, None], wcls[:, None] * (prob - onehot) / b, 0.0)
    ce = (np.log(se[:, 0]) + mx[:, 0] - lg[np.arange(b), np.maximum(label, 0)])
    loss = loss + np.where(has, wcls * ce, 0.0)
    return float(loss.mean()), d


def mlp_backward(x, params, dout, mu=None, sd=None):
    """Gradient of sum(dout * out) w.r.t. the packed parameters (float64).  The
    weight matrices enter the forward pass rounded to bf16; the gradient is taken
    with respect to those rounded values (straight-through), as the CUDA kernels do."""
    p = unpack(params)
    xn, h1, h2, _ = mlp_forward(x, params, mu, sd)
    w2, w3 = (bf16(p[k]).astype(np.float64) for k in ("W2", "W3"))
    dout = np.asarray(dout, np.float64)
    g = {"W3": h2.T @ dout, "b3": dout.sum(0)}
    dh2 = (dout @ w3.T) * (h2 > 0)
    g["W2"], g["b2"] = h1.T @ dh2, dh2.sum(0)
    dh1 = (dh2 @ w2.T) * (h1 > 0)
    g["W1"], g["b1"] = xn.T @ dh1, dh1.sum(0)
    out = np.zeros(NPARAMS, dtype=np.float64)
    for k, (o, s) in offsets().items():
        out[o:o + int(np.prod(s))] = g[k].ravel()
    return out


def _mix64(x):
    x = (x + 0x9E3779B97F4A7C15) & _M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _M64
    return x ^ (x >> 31)


def _slog2(x):
    return np.log2(1.0 + x) if x >= 0 else -np.log2(1.0 - x)


def sketch(keys, valid=None, n=None):
    """280 float32 features of the first min(n, 65536) rows (keys: int32 array)."""
    keys = np.asarray(keys, dtype=np.int32)
    n = keys.size if n is None else int(n)
    m = min(n, SKETCH_ROWS)
    k = keys[:m].astype(np.int64)
    v = np.ones(m, bool) if valid is None else np.asarray(valid[:m], bool)
    kv = k[v]
    regs = np.zeros(REGS, dtype=np.int64)
    for key in kv.tolist():
        h = _mix64(key & 0xFFFFFFFF)
        idx = h >> 56
        rest = ((h << 8) & _M64) | 0x80
        r = min(64 - rest.bit_length() + 1, 57)
        if r > regs[idx]:
            regs[idx] = r
    feat = np.zeros(IN, dtype=np.float32)
    feat[:REGS] = (regs / 16.0).astype(np.float32)
    if kv.size:
        kmin, kmax, first = int(kv.min()), int(kv.max()), int(kv[0])
        span = float(kmax - kmin) + 1.0
    else:
        kmin = kmax = first = 0
        span = 0.0
    t = np.zeros(16, dtype=np.float64)
    t[0] = kv.size
    t[1] = np.count_nonzero(kv == first)
    pos = (kv.astype(np.float64) - kmin) / span if span > 0 else np.zeros(kv.size)
    t[2] = np.count_nonzero(pos < 0.5)
    t[3] = np.count_nonzero(pos < 0.0625)
    pair = v[:-1] & v[1:]
    d = (k[1:] - k[:-1])[pair]
    ad = np.abs(d)
    t[4] = d.size
    t[5] = np.count_nonzero(d == 0)
    t[6] = np.count_nonzero(d > 0)
    t[7] = np.count_nonzero(d < 0)
    t[8] = np.count_nonzero(ad < 1024)
    t[9] = np.count_nonzero(ad < 65536)
    ku = k.astype(np.uint32)
    t[10] = np.count_nonzero(((ku[:-1] >> 16) == (ku[1:] >> 16))[pair])
    t[11] = int(np.sum(np.minimum(ad, 1 << 40) >> 8))
    if m > 8:
        p8 = v[:-8] & v[8:]
        t[12] = np.count_nonzero(p8)
        t[13] = np.count_nonzero((k[8:] == k[:-8])[p8])
    t[14] = np.count_nonzero((k[1:] != k[:-1])[pair])
    z = float(np.sum(np.ldexp(1.0, -regs)))
    zeros = int(np.count_nonzero(regs == 0))
    mm = float(REGS)
    est = 0.7182725932 * mm * mm / z
    if est <= 2.5 * mm and zeros > 0:
        est = mm * np.log(mm / zeros)
    valid_n = t[0]
    pairs = t[4] if t[4] > 0 else 1.0
    heads = t[14] + 1.0
    st = [np.log2(1.0 + n) / 32.0, np.log2(1.0 + m) / 17.0, valid_n / m if m > 0 else 0.0,
          np.log2(1.0 + est) / 32.0, zeros / REGS, t[5] / pairs, np.log2(1.0 + valid_n / heads) / 17.0,
          t[13] / t[12] if t[12] > 0 else 0.0, t[6] / pairs, t[7] / pairs, np.log2(1.0 + span) / 32.0,
          1.0 if kmin >= 0 else 0.0, _slog2(float(kmin)) / 32.0, _slog2(float(kmax)) / 32.0,
          (np.log2(1.0 + span) - np.log2(1.0 + valid_n)) / 32.0, np.log2(1.0 + 256.0 * t[11] / pairs) / 40.0,
          t[8] / pairs, t[9] / pairs, t[2] / valid_n if valid_n > 0 else 0.0,
          t[3] / valid_n if valid_n > 0 else 0.0, t[1] / valid_n if valid_n > 0 else 0.0,
          min(est / valid_n, 4.0) if valid_n > 0 else 0.0, np.log2((1.0 + n) / (1.0 + m)) / 16.0, t[10] / pairs]
    feat[REGS:] = np.asarray(st, dtype=np.float64).astype(np.float32)
    return feat


def plan_fixed_class(n, span, kmin, naggs, is_sorted):
    """The reference rule's class for a probe: 'sorted', 'dense' or 'hash'
    (src/Runtime/Planner/_lib/planner.py:200-262 with groupindex.py:72-83 estimates and
    the 2^31 - 1 byte budget)."""
    if n == 0:
        return "empty"
    if is_sorted:
        return "sorted"
    cap = min(64_000_000, 4 * n)
    naggs = max(1, naggs)
    total_shift = 16 * span + 8 * n + naggs * (8 * min(span, n) + 8 * n)
    budget = 2 ** 31 - 1
    if kmin >= 0:
        m = kmin + span
        total_code = 16 * m + 8 * n + naggs * 8 * min(m, n)
        if m <= cap and total_code <= budget and total_code <= total_shift:
            return "dense"
    if span <= cap and total_shift <= budget:
        return "dense"
    return "hash"
