"""LDPC code descriptions: the parity-check matrix H as check rows in layer order.

The reference compiles one H matrix into the binary (``src/matrix/code.h:1``
selects it; ``src/matrix/<code>/constantes_decoder.h`` holds the flattened
check-major variable-index list ``PosNoeudsVariable[_M]``).  Here a code is a
runtime object: rows in the decoder's layer order, each a list of variable
indices, loaded from the shipped ``codes/*.ldpc`` tables (converted once from
the reference tables by ``codes/import_reference_tables.py``) or built by the
generators in this module.

Row "class": the reference groups rows into at most two degree classes
(``DEG_1`` rows first, then ``DEG_2`` rows); the offset-min-sum kernel treats
the second group differently in the first iteration
(``decoder_oms/cuda/CUDA_OMS_SIMD.cu:115-116``), so each row records which
group it came from.
"""
import os
import struct

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
TABLE_DIR = os.path.join(_HERE, "codes")
MAGIC = b"LDPCH001"


class Code:
    """Parity-check matrix as CSR rows (row order = layer order).

    Attributes: ``name``, ``n`` (variables), ``m`` (checks), ``e`` (edges),
    ``row_ptr`` (int32, m+1), ``cols`` (int32, e), ``row_class`` (uint8, m).
    ``n_info`` = n - m, the number of bits the reference's error analyser
    counts per frame (``trame/CTrame.cpp:65-67``).
    """

    def __init__(self, name, n, row_ptr, cols, row_class=None):
        self.name = name
        self.n = int(n)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.m = len(self.row_ptr) - 1
        self.e = int(self.row_ptr[-1])
        if row_class is None:
            row_class = np.zeros(self.m, dtype=np.uint8)
        self.row_class = np.ascontiguousarray(row_class, dtype=np.uint8)
        if self.e != len(self.cols):
            raise ValueError("row_ptr/cols mismatch")
        if self.e and (self.cols.min() < 0 or self.cols.max() >= self.n):
            raise ValueError("column index out of range")

    @property
    def n_info(self):
        return self.n - self.m

    @property
    def degrees(self):
        return np.diff(self.row_ptr)

    def rows(self):
        for r in range(self.m):
            yield self.cols[self.row_ptr[r]:self.row_ptr[r + 1]]

    def dense(self):
        h = np.zeros((self.m, self.n), dtype=np.uint8)
        for r, c in enumerate(self.rows()):
            h[r, c] ^= 1
        return h

    def syndrome(self, bits):
        """Per-frame parity checks of hard decisions ``bits`` [frames, n] (0/1)."""
        bits = np.asarray(bits, dtype=np.uint8)
        s = np.zeros((bits.shape[0], self.m), dtype=np.uint8)
        for r, c in enumerate(self.rows()):
            s[:, r] = np.bitwise_xor.reduce(bits[:, c], axis=1)
        return s

    @classmethod
    def from_groups(cls, name, n, groups, cols):
        """Rows of uniform degree in consecutive groups [(degree, count), ...]."""
        row_ptr = [0]
        row_class = []
        for gi, (d, c) in enumerate(groups):
            for _ in range(c):
                row_ptr.append(row_ptr[-1] + d)
                row_class.append(min(gi, 1))
        return cls(name, n, np.array(row_ptr), cols, np.array(row_class, dtype=np.uint8))

    @classmethod
    def from_rows(cls, name, n, rows, row_class=None):
        row_ptr = np.zeros(len(rows) + 1, dtype=np.int64)
        row_ptr[1:] = np.cumsum([len(r) for r in rows])
        cols = np.concatenate([np.asarray(r, dtype=np.int64) for r in rows]) if rows else np.zeros(0)
        return cls(name, n, row_ptr, cols, row_class)

    @classmethod
    def from_file(cls, path, name=None):
        b = open(path, "rb").read()
        if b[:8] != MAGIC:
            raise ValueError("not an .ldpc table: %s" % path)
        n, k, m, ng, cb, _ = struct.unpack_from("<6I", b, 8)
        off = 32
        groups = [struct.unpack_from("<2I", b, off + 8 * i) for i in range(ng)]
        off += 8 * ng
        cols = np.frombuffer(b, dtype=np.uint16 if cb == 2 else np.uint32, count=m, offset=off)
        code = cls.from_groups(name or os.path.splitext(os.path.basename(path))[0], n, groups, cols)
        if code.m != k:
            raise ValueError("table check count mismatch")
        code.groups = groups
        return code

    def to_file(self, path):
        """Writes the table format; rows must form consecutive uniform-degree groups."""
        groups = []
        deg = self.degrees
        for d in deg:
            if groups and groups[-1][0] == d:
                groups[-1][1] += 1
            else:
                groups.append([int(d), 1])
        cb = 2 if self.n <= 65536 else 4
        with open(path, "wb") as f:
            f.write(MAGIC)
            f.write(struct.pack("<6I", self.n, self.m, self.e, len(groups), cb, 0))
            for d, c in groups:
                f.write(struct.pack("<2I", d, c))
            f.write(self.cols.astype(np.uint16 if cb == 2 else np.uint32).tobytes())


# ---------------------------------------------------------------------------
# generators (no reference counterpart: the reference only ships fixed tables)
# ---------------------------------------------------------------------------

def _qc_has_4cycle(base, shifts, z, i, j):
    """True if the nonzero (i, j) closes a 4-cycle with already-assigned entries:
    s(i,j) - s(i,j') + s(i',j') - s(i',j) = 0 (mod z) for some rows i' and columns j'."""
    rows = np.flatnonzero(base[:, j])
    cols = np.flatnonzero(base[i, :])
    for i2 in rows:
        if i2 == i:
            continue
        for j2 in cols:
            if j2 == j or not base[i2, j2]:
                continue
            if (shifts[i, j] - shifts[i, j2] + shifts[i2, j2] - shifts[i2, j]) % z == 0:
                return True
    return False


def qc_from_base(name, base, shifts, z):
    """Expands a base matrix (0/1) with circulant shifts into H.  Block row i, row k
    of the block connects to variable j*z + (k + s_ij) mod z for every nonzero (i, j);
    one block row is one layer (its z rows share no variable)."""
    mb, nb = base.shape
    rows = []
    for i in range(mb):
        js = np.flatnonzero(base[i])
        for k in range(z):
            rows.append([j * z + (k + shifts[i, j]) % z for j in js])
    return Code.from_rows(name, nb * z, rows)


def qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name=None):
    """Seeded regular (wc, wr) QC-LDPC code: an mb x nb base matrix with wc nonzeros per
    column at seeded rows and nb*wc/mb per row, circulant shifts uniform in [0, z), and
    4-cycles rejected.  Defaults: (3,6), 8x16, Z=256 -> N=4096, 2048 checks."""
    rng = np.random.default_rng(seed)
    wr = nb * wc // mb
    if wr * mb != nb * wc:
        raise ValueError("not a regular degree pair")
    while True:
        slots = np.repeat(np.arange(mb), wr)
        rng.shuffle(slots)
        cols = slots.reshape(nb, wc)
        if all(len(set(c)) == wc for c in cols):
            break
    base = np.zeros((mb, nb), dtype=np.uint8)
    for j in range(nb):
        base[cols[j], j] = 1
    shifts = np.zeros((mb, nb), dtype=np.int64)
    for j in range(nb):
        for i in np.flatnonzero(base[:, j]):
            for _ in range(10000):
                shifts[i, j] = rng.integers(0, z)
                if not _qc_has_4cycle(base, shifts, z, i, j):
                    break
            else:
                raise RuntimeError("could not avoid 4-cycles")
    code = qc_from_base(name or "qc%dx%d_z%d_s%d" % (mb, nb, z, seed), base, shifts, z)
    code.base, code.shifts, code.z = base, shifts, z
    return code


def ira(n=64800, k=32400, group=360, frac_high=0.2, deg_high=8, deg_low=3, seed=2025, name=None, layered=True):
    """Seeded IRA code (DVB-S2-like structure): information columns in groups of
    `group`; a fraction `frac_high` of the groups have degree `deg_high`, the rest
    `deg_low`; each group's first column draws its check rows uniformly from the
    seed (with distinct residues mod q when q allows) and the other columns of the
    group follow with a cyclic step of q = (n - k) / group, as in DVB-S2.  The
    parity part is the dual-diagonal staircase (parity j in checks j and j+1).
    Defaults: N=64800, K=32400, 1/5 of the groups of degree 8, the rest of degree
    3 (check degree about 6).

    With `layered` the checks are listed in the order i + j*q (i = 0..q-1 outer,
    j = 0..group-1 inner): the `group` checks of one i share no parity bit and,
    because a group's base rows have distinct residues mod q, no information
    bit, so the row-layered decoder runs each such layer in parallel.  In
    natural order consecutive checks share a parity bit and the layered
    schedule is fully serial.  The code is the same; ``code.ira_natural[r]`` is
    the staircase index of row r."""
    m = n - k
    if k % group or m % group:
        raise ValueError("k and n-k must be multiples of the group size")
    q = m // group
    rng = np.random.default_rng(seed)
    ngroups = k // group
    n_high = int(round(frac_high * ngroups))
    rows = [[] for _ in range(m)]
    for gi in range(ngroups):
        deg = deg_high if gi < n_high else deg_low
        # uniform rows with distinct residues mod q (when q allows): a column then
        # meets each layer {i + j*q} at most once
        if deg <= q:
            base = rng.choice(q, size=deg, replace=False) + q * rng.integers(0, group, size=deg)
        else:
            base = rng.choice(m, size=deg, replace=False)
        for c in range(group):
            col = gi * group + c
            for b in base:
                rows[(int(b) + c * q) % m].append(col)
    for j in range(m):
        rows[j].append(k + j)
        if j > 0:
            rows[j].append(k + j - 1)
    rows = [sorted(set(r)) for r in rows]
    natural = np.arange(m)
    if layered:
        natural = (np.arange(q)[:, None] + q * np.arange(group)[None, :]).reshape(-1)
        rows = [rows[j] for j in natural]
    code = Code.from_rows(name or "ira%dx%d_s%d%s" % (n, m, seed, "" if layered else "_nat"), n, rows)
    code.ira_k = k
    code.ira_natural = natural
    return code


class IRAEncoder:
    """Linear-time systematic encoder of an `ira` code: p_j = p_{j-1} + (sum of the
    information bits of check j), i.e. a cumulative XOR down the staircase.  The
    information part of H is kept sparse (one gather and one segmented XOR per
    batch), so N = 64800 codes encode without a dense m x k matrix."""

    def __init__(self, code):
        self.n, self.k = code.n, code.ira_k
        m = code.m
        natural = np.asarray(getattr(code, "ira_natural", np.arange(m)))
        rp = np.asarray(code.row_ptr, dtype=np.int64)
        cols = np.asarray(code.cols, dtype=np.int64)
        nat_of_edge = np.repeat(natural, np.diff(rp))   # staircase index of each edge's check
        keep = cols < self.k
        order = np.argsort(nat_of_edge[keep], kind="stable")
        self.cols = cols[keep][order]
        counts = np.bincount(nat_of_edge[keep], minlength=m)
        self.starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
        self.empty = counts == 0

    def encode(self, info):
        info = np.asarray(info, dtype=np.uint8)
        g = info[:, self.cols]
        s = np.bitwise_xor.reduceat(g, np.minimum(self.starts, g.shape[1] - 1), axis=1)
        s[:, self.empty] = 0
        par = np.bitwise_xor.accumulate(s, axis=1)
        return np.concatenate([info, par], axis=1)


def qc_irregular(z=27, rate=(1, 2), seed=2026, nb=24, degrees=(2, 3, 4, 11), name=None):
    """Seeded irregular QC code with a 24-column base and a dual-diagonal parity part
    (802.11n-like layout): mb = nb*(1-rate) block rows, information block columns of
    degrees drawn from `degrees` (at least one of the largest), a first parity column
    of weight 3 (shifts s, 0, s at the top, middle and bottom rows) and a staircase of
    identity blocks; shifts uniform in [0, z) with 4-cycles rejected."""
    num, den = rate
    mb = nb * (den - num) // den
    kb = nb - mb
    for attempt in range(100):
        rng = np.random.default_rng(seed + 7717 * attempt)
        base = np.zeros((mb, nb), dtype=np.uint8)
        shifts = np.zeros((mb, nb), dtype=np.int64)
        top = min(max(degrees), mb)
        degs = [top] + [min(int(rng.choice(degrees)), mb) for _ in range(kb - 1)]
        for j, d in enumerate(degs):
            base[rng.choice(mb, size=d, replace=False), j] = 1
        # parity part: column kb weight 3 (rows 0, mb//2, mb-1), then the identity staircase;
        # its shifts are fixed first so that the information shifts are checked against them
        for i in (0, mb // 2, mb - 1):
            base[i, kb] = 1
        for j in range(1, mb):
            base[j - 1, kb + j] = 1
            base[j, kb + j] = 1
        s0 = int(rng.integers(1, z))
        for i in (0, mb - 1):
            shifts[i, kb] = s0
        ok = True
        for j in range(kb):
            for i in np.flatnonzero(base[:, j]):
                for _ in range(2000):
                    shifts[i, j] = rng.integers(0, z)
                    if not _qc_has_4cycle(base, shifts, z, i, j):
                        break
                else:
                    ok = False
                    break
            if not ok:
                break
        if ok:
            break
    else:
        raise RuntimeError("no 4-cycle-free base found for z=%d rate %d/%d" % (z, num, den))
    code = qc_from_base(name or "qcirr_z%d_r%d%d_s%d" % (z, num, den, seed), base, shifts, z)
    code.base, code.shifts, code.z = base, shifts, z
    return code


class Encoder:
    """Systematic encoder for any H: Gaussian elimination over GF(2) gives pivot
    (parity) columns P and free (information) columns I with H_P^-1 H_I = A, so a
    codeword is x_I = u, x_P = A u (mod 2)."""

    def __init__(self, code):
        h = code.dense().astype(np.uint8)
        m, n = h.shape
        words = (n + 63) // 64
        packed = np.zeros((m, words), dtype=np.uint64)
        for w in range(words):
            blk = h[:, 64 * w: 64 * w + 64]
            weights = (np.uint64(1) << np.arange(blk.shape[1], dtype=np.uint64))
            packed[:, w] = (blk.astype(np.uint64) * weights).sum(axis=1, dtype=np.uint64)
        pivots = []
        row = 0
        for col in range(n):
            if row == m:
                break
            w, b = divmod(col, 64)
            bit = (packed[row:, w] >> np.uint64(b)) & np.uint64(1)
            nz = np.flatnonzero(bit)
            if nz.size == 0:
                continue
            p = row + nz[0]
            if p != row:
                packed[[row, p]] = packed[[p, row]]
            hits = np.flatnonzero((packed[:, w] >> np.uint64(b)) & np.uint64(1))
            hits = hits[hits != row]
            packed[hits] ^= packed[row]
            pivots.append(col)
            row += 1
        self.rank = row
        self.pivots = np.array(pivots, dtype=np.int64)
        mask = np.ones(n, dtype=bool)
        mask[self.pivots] = False
        self.info_cols = np.flatnonzero(mask)
        red = np.zeros((self.rank, n), dtype=np.uint8)
        for w in range(words):
            chunk = packed[:self.rank, w]
            for b in range(min(64, n - 64 * w)):
                red[:, 64 * w + b] = ((chunk >> np.uint64(b)) & np.uint64(1)).astype(np.uint8)
        self.A = red[:, self.info_cols].astype(np.float32)  # rank x k
        self.n = n
        self.k = n - self.rank

    def encode(self, info):
        """info: [frames, k] 0/1 -> codewords [frames, n] 0/1."""
        info = np.asarray(info, dtype=np.float32)
        par = np.mod(info @ self.A.T, 2.0).astype(np.uint8)
        cw = np.zeros((info.shape[0], self.n), dtype=np.uint8)
        cw[:, self.info_cols] = info.astype(np.uint8)
        cw[:, self.pivots] = par
        return cw


def reference_tables():
    """Names of the shipped tables converted from the reference's src/matrix."""
    return sorted(f[:-5] for f in os.listdir(TABLE_DIR) if f.endswith(".ldpc"))


def load_table(name):
    """Loads a shipped table by name, e.g. ``load_table("4000x2000")``."""
    return Code.from_file(os.path.join(TABLE_DIR, name + ".ldpc"), name)
