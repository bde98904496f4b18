"""Reading the solver's .dat output and the oracle's raw field dumps."""
import numpy as np


def _is_num(tok):
    try:
        float(tok)
        return True
    except ValueError:
        return False


def dat_blocks(path):
    """Split a .dat file into (header_text, array) blocks: every run of
    all-numeric lines after a text line.  Header lines 0-16 (standard) carry
    text and numbers on one line; they are returned as text blocks."""
    with open(path) as f:
        lines = f.read().splitlines()
    blocks = []
    title, rows = None, []
    for ln in lines:
        toks = ln.split()
        if toks and all(_is_num(t) for t in toks):
            if rows and len(toks) != len(rows[-1]):  # e.g. the theta,phi line before a series
                blocks.append((title, np.array(rows)))
                title, rows = title + " (cont.)", []
            rows.append([float(t) for t in toks])
        else:
            if rows:
                blocks.append((title, np.array(rows)))
            title, rows = ln.strip(), []
    if rows:
        blocks.append((title, np.array(rows)))
    return blocks, lines


def header_values(lines, n=17):
    """Numeric tokens of the fixed header lines."""
    out = []
    for ln in lines[:n]:
        out.append([t for t in ln.split() if _is_num(t)])
    return out


def read_oracle_dump(path, kmax=False):
    """Fields written by the oracle with ORACLE_DUMP=path: Ex,Ey,Ez,Hx,Hy,Hz,
    each as int32 dims[3] then float64 values (re,im pairs for kmax), first
    index fastest.  Returned as arrays of shape (nz, ny, nx)."""
    out = []
    with open(path, "rb") as f:
        for _ in range(6):
            dims = np.frombuffer(f.read(12), dtype=np.int32)
            n = int(np.prod(dims))
            v = np.frombuffer(f.read(8 * n * (2 if kmax else 1)), dtype=np.float64)
            if kmax:
                v = v[0::2] + 1j * v[1::2]
            out.append(v.reshape(dims[2], dims[1], dims[0]))
    return out


def rel_l2(a, b, floor=0.0):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.linalg.norm(a), floor)
    if den == 0:
        return float(np.linalg.norm(a - b))
    return float(np.linalg.norm(a - b) / den)
