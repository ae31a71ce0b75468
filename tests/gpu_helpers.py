"""Helpers shared by the GPU parity tests (CPU-side expectation building)."""
import numpy as np


def to_dev(x, dev):
    import torch

    v = x.view(np.int64) if x.dtype == np.uint64 else x.view(np.int32)
    return torch.from_numpy(np.ascontiguousarray(v)).to(dev)


def to_np(t, s):
    a = t.cpu().numpy()
    return a.view(np.uint64) if s == 8 else a.view(np.uint32)


def expected_gpu_column(orc, codec, x, bs):
    """Oracle (= reference) block images with this library's one deliberate
    difference: a block the reference would write with l == 8*sizeof(T)-1
    (LeCo, FOR, poly) is written raw, because the reference's own bulk decoder
    reads l >= 8*sizeof(T)-1 as raw."""
    s = x.dtype.itemsize
    n = len(x)
    nb = (n + bs - 1) // bs
    parts, offs, pos, h1 = [], [], 0, 0
    for b in range(nb):
        blk = x[b * bs:(b + 1) * bs]
        img = orc.encode_block(codec, blk)
        if codec != 2 and img[0] == 8 * s - 1:
            img = bytes([8 * s]) + blk.tobytes()
            h1 += 1
        offs.append(pos)
        parts.append(img)
        pos += len(img)
    offs.append(pos)
    return np.frombuffer(b"".join(parts), np.uint8), np.array(offs, np.uint64), h1


def mask_delta_last_fields(payload, offsets, s, n, bs):
    """Clears the last field of each packed Delta block (the reference writes
    out-of-bounds memory there, delta_integer_template.h:83)."""
    p = payload.copy()
    nb = len(offsets) - 1
    for b in range(nb):
        o = int(offsets[b])
        l = int(p[o])
        m = min(bs, n - b * bs)
        if m < 2 or l in (0, 8 * s):
            continue
        for bit in range((m - 1) * l, m * l):
            p[o + 1 + s + bit // 8] &= ~(1 << (bit % 8)) & 0xFF
    return p
