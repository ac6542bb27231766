"""GIP on-disk formats: binary CSR operators, binary scalar fields and text topologies.

Layouts (recovered from GIP's readers):

* ``.csr`` -- ``GIP_MatrixMulticore::postConstruct`` (src/Specifications/Multicore/
  GIP_MatrixMulticore.cpp:5-31): ``int32 header[5] = {nnz, ncols, nrows,
  ceil(nrows/1024), 1024}``, then ``float64 val[nnz]``, ``int32 col[nnz]``,
  ``int32 rowptr[nrows+1]``; 0-based, rows need not be column-sorted.
* ``.vec`` -- ``GIP_VectorMulticore::postConstruct`` (GIP_VectorMulticore.cpp:26-42):
  ``int32 n`` then ``float64 x[n]``.
* ``.topo`` -- ``GIP_Topo::postConstruct`` (src/BasicInterfaces/GIP_Topo.cpp:3-57): nine
  whitespace-separated integers ``send_size recv_size cols_size owned all interiors
  interfaces boundaries halos`` then ``send_indx[send_size]``, ``send_row[cols_size]``,
  ``recv_indx[recv_size]``, ``recv_row[cols_size]``.  Cells of a rank are laid out
  ``[interiors | interfaces | boundaries | halos]`` (GIP_Topo.h:8-18).

File naming follows ``GIP_DNS::upload*`` (src/Algorithms/GIP_DNS.h:143-306):
``InputFiles/Operators/<grp>/<case>/<case>_<np>p/<Op><case>_<np>p-<rank>.csr`` and the
matching ``Scalarfields`` / ``Topos`` trees.

Besides plain I/O this module merges an ``np``-rank operator set into one global
single-rank set (the drop-in runs at one rank) and splits a single-rank set into
``np`` slab ranks so GIP's own MPI CPU build can run the same operators.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

# operator name -> InputFiles/Operators/<group>
OPERATOR_GROUPS: Dict[str, str] = {
    "D": "CD", "Ec": "CD",
    "L": "L", "Lb": "L",
    "Mx": "M", "My": "M", "Mz": "M", "Mres": "M",
    "Gx": "G", "Gy": "G", "Gz": "G",
    "SFx": "S", "SFy": "S", "SFz": "S", "SO": "S",
}
FIELD_NAMES = ("u", "v", "w", "dxs")

# row space / column space of every operator ("cell", "face" or "dnnz" = one row per
# nonzero of D, the layout of Ec whose product is C's value array, GIP_DNS.h:312)
OPERATOR_SPACES: Dict[str, tuple] = {
    "D": ("inner", "cell"), "L": ("inner", "cell"), "Lb": ("owned", "cell"),
    "Mx": ("inner", "cell"), "My": ("inner", "cell"), "Mz": ("inner", "cell"),
    "Mres": ("inner", "face"),
    "Gx": ("owned", "cell"), "Gy": ("owned", "cell"), "Gz": ("owned", "cell"),
    "SFx": ("face", "cell"), "SFy": ("face", "cell"), "SFz": ("face", "cell"),
    "SO": ("face", "cell"),
    "Ec": ("dnnz", "face"),
}


class FormatError(ValueError):
    """A GIP file is truncated, inconsistent or out of range."""


@dataclasses.dataclass
class Csr:
    nrows: int
    ncols: int
    rowptr: np.ndarray  # int32 [nrows+1]
    col: np.ndarray     # int32 [nnz]
    val: np.ndarray     # float64 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def validate(self, name: str = "csr", col_bound: Optional[int] = None) -> None:
        """Check rowptr monotonicity and, when ``col_bound`` is given, column range.
        The header's ``ncols`` is not a bound: GIP's per-rank operators reference halo
        cells past the owned range (e.g. C100K_4p D: ncols=26235, halo columns above)."""
        rp = self.rowptr
        if rp.shape != (self.nrows + 1,):
            raise FormatError(f"{name}: rowptr has {rp.shape[0]} entries, want {self.nrows + 1}")
        if self.nrows and (rp[0] != 0 or np.any(np.diff(rp.astype(np.int64)) < 0)):
            raise FormatError(f"{name}: rowptr is not monotone from 0")
        if int(rp[-1]) != self.nnz or self.val.shape[0] != self.nnz:
            raise FormatError(f"{name}: rowptr[-1]={int(rp[-1])} but nnz={self.nnz}")
        if self.nnz and int(self.col.min()) < 0:
            raise FormatError(f"{name}: negative column index")
        if col_bound is not None and self.nnz and int(self.col.max()) >= col_bound:
            raise FormatError(f"{name}: column index out of [0,{col_bound})")

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.rowptr), shape=(self.nrows, self.ncols))

    def copy(self) -> "Csr":
        return Csr(self.nrows, self.ncols, self.rowptr.copy(), self.col.copy(), self.val.copy())


@dataclasses.dataclass
class Topo:
    owned: int
    all: int
    interiors: int
    interfaces: int
    boundaries: int
    halos: int
    send_indx: np.ndarray
    send_row: np.ndarray
    recv_indx: np.ndarray
    recv_row: np.ndarray

    @property
    def inner(self) -> int:
        return self.interiors + self.interfaces

    @property
    def cols_size(self) -> int:
        return int(self.send_row.shape[0])

    @staticmethod
    def single_rank(owned: int, inner: int, boundaries: int) -> "Topo":
        """Topology of a one-rank run: no halo, ``cols_size`` 2 with empty send/recv."""
        z = np.zeros(2, np.int32)
        return Topo(owned, owned, inner, 0, boundaries, 0,
                    np.zeros(0, np.int32), z.copy(), np.zeros(0, np.int32), z.copy())


@dataclasses.dataclass
class GipCase:
    """One rank's operators, initial fields and topologies."""
    ops: Dict[str, Csr]
    fields: Dict[str, np.ndarray]
    topo_cols: Topo
    topo_faces: Topo
    # global id of every local cell (split_ranks sets it: local cell k is global cell_ids[k])
    cell_ids: Optional[np.ndarray] = None

    @property
    def n_inner(self) -> int:
        return self.topo_cols.inner

    @property
    def n_owned(self) -> int:
        return self.topo_cols.owned

    @property
    def n_faces(self) -> int:
        return self.topo_faces.all


# ----------------------------------------------------------------------------- raw I/O
def read_csr(path: str) -> Csr:
    with open(path, "rb") as f:
        buf = f.read()
    if len(buf) < 20:
        raise FormatError(f"{path}: shorter than the 20-byte header")
    nnz, ncols, nrows = (int(x) for x in np.frombuffer(buf[:20], np.int32)[:3])
    if nnz < 0 or ncols < 0 or nrows < 0:
        raise FormatError(f"{path}: negative size in header")
    need = 20 + 12 * nnz + 4 * (nrows + 1)
    if len(buf) < need:
        raise FormatError(f"{path}: {len(buf)} bytes, header implies {need}")
    o = 20
    val = np.frombuffer(buf, np.float64, nnz, o).copy(); o += 8 * nnz
    col = np.frombuffer(buf, np.int32, nnz, o).copy(); o += 4 * nnz
    rowptr = np.frombuffer(buf, np.int32, nrows + 1, o).copy()
    m = Csr(nrows, ncols, rowptr, col, val)
    m.validate(path)
    return m


def write_csr(path: str, m: Csr) -> None:
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    hdr = np.array([m.nnz, m.ncols, m.nrows, (m.nrows + 1023) // 1024, 1024], np.int32)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.ascontiguousarray(m.val, np.float64).tobytes())
        f.write(np.ascontiguousarray(m.col, np.int32).tobytes())
        f.write(np.ascontiguousarray(m.rowptr, np.int32).tobytes())


def read_vec(path: str, size: Optional[int] = None) -> np.ndarray:
    with open(path, "rb") as f:
        buf = f.read()
    if len(buf) < 4:
        raise FormatError(f"{path}: missing length")
    n = int(np.frombuffer(buf[:4], np.int32)[0])
    if n < 0 or len(buf) < 4 + 8 * n:
        raise FormatError(f"{path}: length {n} does not match file size {len(buf)}")
    x = np.frombuffer(buf, np.float64, n, 4).copy()
    if size is not None and n < size:
        # GIP reads `n` values into a vector of `allsize` (GIP_VectorMulticore.cpp:46-48);
        # the rest is left as allocated.  Zero-extend.
        x = np.concatenate([x, np.zeros(size - n)])
    return x


def write_vec(path: str, x: np.ndarray) -> None:
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "wb") as f:
        f.write(np.array([x.shape[0]], np.int32).tobytes())
        f.write(np.ascontiguousarray(x, np.float64).tobytes())


def read_topo(path: str) -> Topo:
    with open(path) as f:
        t = [int(x) for x in f.read().split()]
    if len(t) < 9:
        raise FormatError(f"{path}: fewer than 9 header integers")
    ss, rs, cs, owned, alls, inter, iface, bnd, halo = t[:9]
    need = 9 + ss + cs + rs + cs
    if len(t) < need:
        raise FormatError(f"{path}: {len(t)} integers, header implies {need}")
    o = 9
    si = np.array(t[o:o + ss], np.int32); o += ss
    sr = np.array(t[o:o + cs], np.int32); o += cs
    ri = np.array(t[o:o + rs], np.int32); o += rs
    rr = np.array(t[o:o + cs], np.int32)
    return Topo(owned, alls, inter, iface, bnd, halo, si, sr, ri, rr)


def write_topo(path: str, t: Topo) -> None:
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    def line(a):
        return " " + " ".join(str(int(v)) for v in a) + " \n"
    hdr = [t.send_indx.shape[0], t.recv_indx.shape[0], t.cols_size, t.owned, t.all,
           t.interiors, t.interfaces, t.boundaries, t.halos]
    with open(path, "w") as f:
        f.write(line(hdr) + line(t.send_indx) + line(t.send_row) + line(t.recv_indx) +
                line(t.recv_row))


# ----------------------------------------------------------------------------- case paths
def op_path(root: str, case: str, nparts: int, rank: int, op: str) -> str:
    grp = OPERATOR_GROUPS[op]
    tag = f"{case}_{nparts}p"
    return os.path.join(root, "InputFiles", "Operators", grp, case, tag, f"{op}{tag}-{rank}.csr")


def field_path(root: str, case: str, nparts: int, rank: int, name: str) -> str:
    tag = f"{case}_{nparts}p"
    return os.path.join(root, "InputFiles", "Scalarfields", case, tag, f"{name}{tag}-{rank}.vec")


def topo_path(root: str, case: str, nparts: int, rank: int, kind: str) -> str:
    tag = f"{case}_{nparts}p"
    return os.path.join(root, "InputFiles", "Topos", case, tag, f"topo{kind}{tag}-{rank}.topo")


def load_case(root: str, case: str, nparts: int = 1, rank: int = 0) -> GipCase:
    tc = read_topo(topo_path(root, case, nparts, rank, "Cols"))
    tf = read_topo(topo_path(root, case, nparts, rank, "Faces"))
    ops = {op: read_csr(op_path(root, case, nparts, rank, op)) for op in OPERATOR_GROUPS}
    fields = {n: read_vec(field_path(root, case, nparts, rank, n), tc.all) for n in FIELD_NAMES}
    return GipCase(ops, fields, tc, tf)


def write_case(root: str, case: str, parts: Sequence[GipCase]) -> None:
    nparts = len(parts)
    for r, c in enumerate(parts):
        for op, m in c.ops.items():
            write_csr(op_path(root, case, nparts, r, op), m)
        for n in FIELD_NAMES:
            write_vec(field_path(root, case, nparts, r, n), c.fields[n])
        write_topo(topo_path(root, case, nparts, r, "Cols"), c.topo_cols)
        write_topo(topo_path(root, case, nparts, r, "Faces"), c.topo_faces)


def check_case(c: GipCase) -> None:
    """Cross-check operator shapes against the topologies (host-side validation that the
    reference never does; GIP reads whatever the headers claim)."""
    n_in, n_own, n_all, nf = c.topo_cols.inner, c.topo_cols.owned, c.topo_cols.all, c.topo_faces.all
    space = {"inner": n_in, "owned": n_own, "cell": n_all, "face": nf,
             "dnnz": c.ops["D"].nnz}
    for op, (rs, cs) in OPERATOR_SPACES.items():
        m = c.ops[op]
        m.validate(op, n_all if cs == "cell" else nf)
        if m.nrows > space[rs]:
            raise FormatError(f"{op}: {m.nrows} rows exceed the {rs} space ({space[rs]})")
    if c.ops["Ec"].nrows != c.ops["D"].nnz:
        raise FormatError("Ec must have one row per nonzero of D")
    for n in FIELD_NAMES:
        if c.fields[n].shape[0] != n_all:
            raise FormatError(f"field {n} has {c.fields[n].shape[0]} entries, want {n_all}")


# ----------------------------------------------------------------------------- merge
def merge_ranks(root: str, case: str, nparts: int) -> GipCase:
    """Merge an ``nparts``-rank set into one global single-rank set.

    Global cell order is ``[inner cells of rank 0..np-1 | boundary cells of rank
    0..np-1]``; halo columns are resolved through the sender's ``send_indx`` (the
    exchange ``GIP_Topo::sendrecv`` performs, GIP_Topo.cpp:150-173).  Faces, and
    Ec rows (one per nonzero of D), are concatenated rank by rank, keeping every
    row's nonzero order, so each product sums in the same order as at ``np`` ranks.
    """
    parts = [load_case(root, case, nparts, r) for r in range(nparts)]
    T = [p.topo_cols for p in parts]
    inner = [t.inner for t in T]
    bnd = [t.owned - t.inner for t in T]
    ioff = np.concatenate([[0], np.cumsum(inner)]).astype(np.int64)
    n_inner = int(ioff[-1])
    boff = n_inner + np.concatenate([[0], np.cumsum(bnd)]).astype(np.int64)
    n_owned = int(boff[-1])
    nfaces = [p.topo_faces.all for p in parts]
    foff = np.concatenate([[0], np.cumsum(nfaces)]).astype(np.int64)
    dnnz = [p.ops["D"].nnz for p in parts]
    doff = np.concatenate([[0], np.cumsum(dnnz)]).astype(np.int64)

    gmap = []
    for r, t in enumerate(T):
        g = np.full(t.all, -1, np.int64)
        g[:t.inner] = ioff[r] + np.arange(t.inner)
        g[t.inner:t.owned] = boff[r] + np.arange(t.owned - t.inner)
        for q in range(nparts):
            a, b = int(t.recv_row[q]), int(t.recv_row[q + 1])
            if b <= a:
                continue
            tq = T[q]
            pos = int(tq.send_row[r]) + np.arange(b - a)
            lq = tq.send_indx[pos].astype(np.int64)
            if np.any(lq >= tq.inner):
                raise FormatError("merge: a sent cell is not an inner cell of its rank")
            g[t.recv_indx[a:b]] = ioff[q] + lq
        if np.any(g < 0):
            raise FormatError(f"merge: rank {r} has halo cells no rank sends")
        gmap.append(g)

    def row_index(kind: str, r: int, nr: int) -> np.ndarray:
        i = np.arange(nr, dtype=np.int64)
        if kind in ("inner", "owned"):
            t = T[r]
            return np.where(i < t.inner, ioff[r] + i, boff[r] + (i - t.inner))
        if kind == "face":
            return foff[r] + i
        return doff[r] + i  # dnnz

    space_rows = {"inner": n_inner, "owned": n_owned, "face": int(foff[-1]),
                  "dnnz": int(doff[-1])}
    space_cols = {"cell": n_owned, "face": int(foff[-1])}
    ops: Dict[str, Csr] = {}
    for op, (rk, ck) in OPERATOR_SPACES.items():
        nrows_g = space_rows[rk]
        lens = np.zeros(nrows_g, np.int64)
        chunks = []
        for r, p in enumerate(parts):
            m = p.ops[op]
            rg = row_index(rk, r, m.nrows)
            lens[rg] = np.diff(m.rowptr)
            cg = gmap[r][m.col] if ck == "cell" else foff[r] + m.col
            chunks.append((rg, m, cg))
        rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        col = np.empty(int(rowptr[-1]), np.int64)
        val = np.empty(int(rowptr[-1]), np.float64)
        for rg, m, cg in chunks:
            rl = np.diff(m.rowptr).astype(np.int64)
            dst = np.repeat(rowptr[rg], rl) + (np.arange(m.nnz) - np.repeat(m.rowptr[:-1], rl))
            col[dst] = cg
            val[dst] = m.val
        ops[op] = Csr(nrows_g, space_cols[ck], rowptr.astype(np.int32), col.astype(np.int32), val)

    fields = {}
    for n in FIELD_NAMES:
        out = np.zeros(n_owned)
        for r, p in enumerate(parts):
            t = T[r]
            out[ioff[r]:ioff[r + 1]] = p.fields[n][:t.inner]
            out[boff[r]:boff[r + 1]] = p.fields[n][t.inner:t.owned]
        fields[n] = out
    tc = Topo.single_rank(n_owned, n_inner, n_owned - n_inner)
    nf = int(foff[-1])
    tf = Topo.single_rank(nf, n_inner, n_owned - n_inner)
    return GipCase(ops, fields, tc, tf)


# ----------------------------------------------------------------------------- split
def split_ranks(c: GipCase, cell_part: np.ndarray, nparts: int) -> List[GipCase]:
    """Split a single-rank case into ``nparts`` ranks.

    ``cell_part[i]`` is the rank owning global cell ``i`` (inner and boundary cells).
    A rank's faces are all faces of its inner cells (the columns of its Mres and Ec
    rows), so faces on a partition boundary exist on both ranks, as in GIP's shipped
    per-rank sets.  A rank's local cells are ordered ``[interiors | interfaces |
    boundaries | halos]`` (GIP_Topo.h:8-18); interface cells are inner cells some
    other rank reads, halos are the remote cells this rank reads, grouped by owner
    rank.  Ec rows follow the local D nonzero order.
    """
    n_in, n_own = c.n_inner, c.n_owned
    nf = c.n_faces
    if cell_part.shape[0] != n_own:
        raise ValueError("partition vector does not match the case size")
    cp = cell_part.astype(np.int64)
    D, Ec, Mres = c.ops["D"], c.ops["Ec"], c.ops["Mres"]
    faces_of = []
    for r in range(nparts):
        own_in = np.nonzero(cp[:n_in] == r)[0]
        fc = [Mres.col[_row_nnz_index(Mres.rowptr, own_in[own_in < Mres.nrows])],
              Ec.col[_row_nnz_index(Ec.rowptr, _row_nnz_index(D.rowptr, own_in))]]
        faces_of.append(np.unique(np.concatenate(fc).astype(np.int64)))

    def rows_of(op: str, r: int) -> np.ndarray:
        m = c.ops[op]
        if OPERATOR_SPACES[op][0] == "face":
            fr = faces_of[r]
            return fr[fr < m.nrows]
        return np.nonzero(cp[:m.nrows] == r)[0]

    halos = []
    for r in range(nparts):
        cols = []
        for op, (rk, ck) in OPERATOR_SPACES.items():
            if ck != "cell":
                continue
            m = c.ops[op]
            cols.append(m.col[_row_nnz_index(m.rowptr, rows_of(op, r))])
        rd = np.unique(np.concatenate(cols).astype(np.int64)) if cols else np.zeros(0, np.int64)
        remote = rd[cp[rd] != r]
        if np.any(remote >= n_in):
            raise ValueError("split: a rank reads another rank's boundary cell")
        halos.append(remote[np.lexsort((remote, cp[remote]))])
    all_halo = np.concatenate(halos) if halos else np.zeros(0, np.int64)
    is_iface = np.zeros(n_own, bool)
    is_iface[all_halo] = True

    layouts = []
    for r in range(nparts):
        own_inner = np.nonzero(cp[:n_in] == r)[0]
        interiors = own_inner[~is_iface[own_inner]]
        interfaces = own_inner[is_iface[own_inner]]
        bcells = n_in + np.nonzero(cp[n_in:] == r)[0]
        order = np.concatenate([interiors, interfaces, bcells, halos[r]])
        layouts.append((order, interiors.size, interfaces.size, bcells.size, halos[r].size))

    parts = []
    for r in range(nparts):
        order, ni, nif, nb, nh = layouts[r]
        inner_l, owned_l = ni + nif, ni + nif + nb
        all_l = owned_l + nh
        g2l = np.full(n_own, -1, np.int64)
        g2l[order] = np.arange(all_l)
        fr = faces_of[r]
        f2l = np.full(nf, -1, np.int64)
        f2l[fr] = np.arange(fr.size)
        ops = {}
        for op, (rk, ck) in OPERATOR_SPACES.items():
            m = c.ops[op]
            cmap, ncl = (g2l, all_l) if ck == "cell" else (f2l, fr.size)
            if op == "Ec":
                row_src = _row_nnz_index(D.rowptr, order[:inner_l])
                nrows_l = row_src.size
            elif rk == "face":
                row_src, nrows_l = fr, fr.size
            else:
                nrows_l = inner_l if rk == "inner" else owned_l
                row_src = order[:nrows_l].copy()
                row_src[row_src >= m.nrows] = -1
            ops[op] = _take_rows(m, row_src, nrows_l, cmap, ncl)
        fields = {n: c.fields[n][order] for n in FIELD_NAMES}
        send_idx, send_row = [], [0]
        for q in range(nparts):
            if q != r:
                oq, _, _, _, nhq = layouts[q]
                hq = oq[oq.size - nhq:]
                send_idx.append(g2l[hq[cp[hq] == r]])
            send_row.append(send_row[-1] + (send_idx[-1].size if q != r else 0))
        hal = order[owned_l:]
        recv_idx, recv_row = [], [0]
        for q in range(nparts):
            sel = owned_l + np.nonzero(cp[hal] == q)[0]
            recv_idx.append(sel)
            recv_row.append(recv_row[-1] + sel.size)
        cat = lambda a: np.concatenate(a).astype(np.int32) if a else np.zeros(0, np.int32)
        tc = Topo(owned_l, all_l, ni, nif, nb, nh, cat(send_idx), np.array(send_row, np.int32),
                  cat(recv_idx), np.array(recv_row, np.int32))
        z = np.zeros(nparts + 1, np.int32)
        tf = Topo(fr.size, fr.size, ni, nif, nb, nh, np.zeros(0, np.int32), z,
                  np.zeros(0, np.int32), z.copy())
        parts.append(GipCase(ops, fields, tc, tf, cell_ids=order.copy()))
    return parts


def _row_nnz_index(rowptr: np.ndarray, rows: np.ndarray) -> np.ndarray:
    """Indices of all nonzeros of the given rows, row after row in row order."""
    rp = rowptr.astype(np.int64)
    rows = np.asarray(rows, np.int64)
    lens = rp[rows + 1] - rp[rows]
    total = int(lens.sum())
    if total == 0:
        return np.zeros(0, np.int64)
    starts = np.repeat(rp[rows] - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens)
    return starts + np.arange(total)


def _take_rows(m: Csr, row_src: np.ndarray, nrows_l: int, cmap: np.ndarray,
               ncols_l: int) -> Csr:
    """Gather rows ``row_src`` of ``m`` (``-1`` = empty row) and renumber columns
    through ``cmap`` (global -> local)."""
    rp = m.rowptr.astype(np.int64)
    valid = row_src >= 0
    rs = row_src[valid]
    lens = np.zeros(nrows_l, np.int64)
    lens[np.nonzero(valid)[0]] = rp[rs + 1] - rp[rs]
    idx = _row_nnz_index(m.rowptr, rs)
    cols = cmap[m.col[idx].astype(np.int64)]
    if np.any(cols < 0):
        raise ValueError("split: a column maps outside the rank's cells/faces")
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    return Csr(nrows_l, ncols_l, rowptr, cols.astype(np.int32), m.val[idx].copy())
