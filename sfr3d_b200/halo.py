"""Row-partitioned solves over several GPUs: the reference's MPI path.

The reference splits the mesh among MPI ranks; each rank assembles its rows
in the MPI CSRD layout (Datastruct.c:129-190) and solverC runs mpiPcg
(Cg.c:256-442) or mpiPbicgstab (Bicgstab.c:298-520), which refresh the ghost
entries of a vector with comunicateNeq (ParallelMpi.c:3346) before each
product and sum each dot over the ranks with MPI_Allreduce.

Here a ``Layout`` is one rank's share (from ``partition`` of a global
system, or the reference's own arrays), a group is the set of ranks that
solve together, and ``DistSystem`` is one rank's partition resident on its
GPU.  ``NcclGroup`` runs one rank per process (launched with torchrun, the
NCCL id handed out through torch.distributed); ``LocalGroup`` holds every
rank in one process on one device.  ``check_interfaces`` verifies, over a
torch.distributed process group, that every rank receives from each
neighbour exactly the values that neighbour sends, in the same order.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import solver as _sv

_P = ctypes.c_void_p
_I32 = ctypes.c_int32


class InterfaceC(ctypes.Structure):
    """sfr_interface: the reference's Interface (include/Mesh.h:212-222)."""
    _fields_ = [("nRcvs", _I32), ("nSends", _I32), ("iaSends", _P), ("iaRcvs", _P),
                ("fMap", _P), ("xb", _P), ("nVizPart", ctypes.c_uint16), ("vizPart", _P)]


class PartSizesC(ctypes.Structure):
    _fields_ = [(n, _I32) for n in ("nEq", "nEqNov", "nAd", "nAdR", "nRcvs", "nSends",
                                     "nVizPart", "ia_len")]


def _lib() -> ctypes.CDLL:
    L = _sv.lib()
    if getattr(L, "_halo_typed", False):
        return L
    L.sfr_part_create.argtypes = [_I32, _P, _P, _I32, _I32, _P, ctypes.POINTER(_P)]
    L.sfr_part_sizes_of.argtypes = [_P, _I32, ctypes.POINTER(PartSizesC)]
    L.sfr_part_fill.argtypes = [_P, _I32, _P, _P, _P, _P, _P, _P, _P, _P]
    L.sfr_part_destroy.argtypes = [_P]
    L.sfr_dist_group_local.argtypes = [_I32, _I32, ctypes.POINTER(_P)]
    L.sfr_dist_nccl_id.argtypes = [_P]
    L.sfr_dist_group_nccl.argtypes = [_I32, _I32, _P, _I32, ctypes.POINTER(_P)]
    L.sfr_dist_group_destroy.argtypes = [_P]
    L.sfr_dist_group_info.argtypes = [_P, _P, _P, _P]
    L.sfr_gpu_dist_create.argtypes = [_P, _I32, _I32, _I32, _I32, _I32, _P, _P, _I32,
                                      ctypes.POINTER(InterfaceC), ctypes.POINTER(_P)]
    L.sfr_gpu_dist_create_storage.argtypes = [_P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P,
                                              _I32, ctypes.POINTER(InterfaceC),
                                              ctypes.POINTER(_P)]
    L.sfr_gpu_dist_set_values.argtypes = [_P, _P, _P]
    L.sfr_gpu_dist_solve.argtypes = [_P, _I32, _P, _I32, _P, _P, ctypes.c_double,
                                     ctypes.c_uint32, _I32, ctypes.POINTER(_sv.SolveInfoC)]
    L.sfr_gpu_dist_destroy.argtypes = [_P]
    L._halo_typed = True
    return L


@dataclass
class Layout:
    """One rank's rows, ghosts and interface, in the reference's arrays.

    ia, ja: the MPI CSRD (unsym: full rows over local columns; sym: the
    strict lower square part in ia[:nEqNov+1] and the ghost columns in
    ia[nEqNov+1:], indexing ja[nAd:]).  src[k]: index in the global al of
    local entry k.  l2g: global equation of each local one (rows, then
    ghosts).  iaSends, iaRcvs, fMap, vizPart: the Interface arrays."""
    rank: int
    unsym: bool
    nEq: int
    nEqNov: int
    nAd: int
    nAdR: int
    ia: np.ndarray
    ja: np.ndarray
    src: np.ndarray
    l2g: np.ndarray
    iaSends: np.ndarray
    iaRcvs: np.ndarray
    fMap: np.ndarray
    vizPart: np.ndarray
    # the reference's storage code of ia/ja (Define.h:407-412): CSRD from
    # `partition`; `as_storage` gives the others
    storage: int = _sv.CSRD

    @property
    def nRcvs(self) -> int:
        return self.nEq - self.nEqNov

    @property
    def nSends(self) -> int:
        return len(self.fMap) - self.nRcvs

    def values(self, al, ad):
        """This rank's al (nAd + nAdR) and ad (nEqNov) from the global arrays."""
        al = np.asarray(al, dtype=np.float64)
        ad = np.asarray(ad, dtype=np.float64)
        return al[self.src].copy(), ad[self.l2g[:self.nEqNov]].copy()

    def rows(self, v):
        """This rank's entries of a global vector (rows only)."""
        return np.asarray(v, dtype=np.float64)[self.l2g[:self.nEqNov]].copy()

    def sends_to(self, n: int) -> np.ndarray:
        """Global equations sent to neighbour vizPart[n], in send order."""
        return self.l2g[self.fMap[self.iaSends[n]:self.iaSends[n + 1]]]

    def receives_from(self, n: int) -> np.ndarray:
        """Global equations received from neighbour vizPart[n], in order."""
        return self.l2g[self.fMap[self.iaRcvs[n]:self.iaRcvs[n + 1]]]

    def interface(self) -> InterfaceC:
        """An sfr_interface over this layout's arrays (keep the layout alive)."""
        return InterfaceC(nRcvs=self.nRcvs, nSends=self.nSends,
                          iaSends=_sv._ptr(self.iaSends), iaRcvs=_sv._ptr(self.iaRcvs),
                          fMap=_sv._ptr(self.fMap), xb=None, nVizPart=len(self.vizPart),
                          vizPart=_sv._ptr(self.vizPart))


def value_count(lay: Layout) -> int:
    """Values of a layout's storage: nAd + nAdR; 2 nAd + nAdR for unsymmetric
    CSRC / CSRCCOO (al | au | ghost values); nEqNov x width for ELLPACK."""
    if lay.storage == _sv.ELLPACK:
        return int(lay.ia[1])
    if lay.storage in (_sv.CSRC, CSRCCOO) and lay.unsym:
        return 2 * lay.nAd + lay.nAdR
    return lay.nAd + lay.nAdR


CSRDCOO, CSRCCOO = 5, 6  # Define.h:411-412


def as_storage(lay: Layout, storage: int, unsym: bool, ia, ja, al, ad):
    """This rank's share of a global system in another of the reference's MPI
    storages (Datastruct.c:115-420), with its values.

    `lay` comes from ``partition(..., unsym=False)`` (the strict-lower square
    part and the ghost columns in CSR) for CSRC, CSRDCOO and CSRCCOO, and from
    ``partition(..., unsym=True)`` (full rows) for ELLPACK.  ia/ja/al are the
    global system's full CSRD rows (all off-diagonals), ad its diagonal;
    `unsym` picks separate upper values (CSRC, CSRCCOO).  Returns (Layout,
    al, ad) for DistSystem.set_values."""
    ia = np.asarray(ia, np.int64)
    ja = np.asarray(ja, np.int64)
    al = np.asarray(al, np.float64)
    n = len(ia) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ia))
    keys = rows * n + ja[: len(rows)]
    order = np.argsort(keys)
    skeys, svals = keys[order], al[: len(rows)][order]

    def A(gi, gj):
        q = np.asarray(gi, np.int64) * n + np.asarray(gj, np.int64)
        pos = np.searchsorted(skeys, q)
        if np.any(pos >= len(skeys)) or np.any(skeys[np.minimum(pos, len(skeys) - 1)] != q):
            raise ValueError("the pattern is not structurally symmetric")
        return svals[pos]

    g = lay.l2g.astype(np.int64)
    adr = np.asarray(ad, np.float64)[g[:lay.nEqNov]].copy()
    fields = {k: getattr(lay, k) for k in ("rank", "nEq", "nEqNov", "src", "l2g", "iaSends",
                                           "iaRcvs", "fMap", "vizPart")}
    if storage == _sv.ELLPACK:
        if not lay.unsym:
            raise ValueError("ELLPACK takes the full-row layout (partition(..., unsym=True))")
        lens = np.diff(lay.ia)
        w = int(lens.max()) if len(lens) else 1
        eja = np.repeat(np.arange(lay.nEqNov, dtype=np.int32), w).reshape(lay.nEqNov, w)
        ea = np.zeros((lay.nEqNov, w))
        for i in range(lay.nEqNov):
            k0, k1 = int(lay.ia[i]), int(lay.ia[i + 1])
            eja[i, : k1 - k0] = lay.ja[k0:k1]
            ea[i, : k1 - k0] = A(np.full(k1 - k0, g[i]), g[lay.ja[k0:k1]])
        out = Layout(unsym=True, nAd=lay.nEqNov * w, nAdR=0,
                     ia=np.array([w, lay.nEqNov * w], np.int32), ja=eja.ravel(),
                     storage=_sv.ELLPACK, **fields)
        return out, ea.ravel(), adr
    if lay.unsym:
        raise ValueError("CSRC and the COO storages take partition(..., unsym=False)")
    if storage == CSRDCOO and unsym:
        raise ValueError("CSRDCOO is symmetric storage")
    n1 = lay.nEqNov + 1
    low_rows = np.repeat(np.arange(lay.nEqNov, dtype=np.int64), np.diff(lay.ia[:n1]))
    low_cols = lay.ja[: lay.nAd].astype(np.int64)
    rect = lay.ia[n1: 2 * n1]
    rect_rows = np.repeat(np.arange(lay.nEqNov, dtype=np.int64), np.diff(rect))
    rect_cols = lay.ja[lay.nAd: lay.nAd + lay.nAdR].astype(np.int64)
    lower = A(g[low_rows], g[low_cols])
    upper = A(g[low_cols], g[low_rows])
    ghost = A(g[rect_rows], g[rect_cols])
    split = storage in (_sv.CSRC, CSRCCOO) and unsym
    vals = np.concatenate([lower, upper, ghost] if split else [lower, ghost])
    new_ia = lay.ia.copy()
    if storage in (CSRDCOO, CSRCCOO):
        new_ia = np.concatenate([lay.ia[: 2 * n1], rect_rows.astype(np.int32)]).astype(np.int32)
    out = Layout(unsym=bool(split), nAd=lay.nAd, nAdR=lay.nAdR, ia=new_ia, ja=lay.ja.copy(),
                 storage=storage, **fields)
    return out, vals, adr


def partition(neq, ia, ja, unsym, nparts, part=None) -> list[Layout]:
    """Split the rows of a global CSRD system among nparts ranks (part[i]:
    rank of row i; None: contiguous blocks balanced by entries)."""
    L = _lib()
    ia, ja = _sv._i32(ia), _sv._i32(ja)
    pa = None if part is None else _sv._i32(part)
    h = _P()
    rc = L.sfr_part_create(int(neq), _sv._ptr(ia), _sv._ptr(ja), int(bool(unsym)),
                           int(nparts), _sv._ptr(pa), ctypes.byref(h))
    if rc != 0:
        raise _sv.SolverError(rc, "sfr_part_create")
    out = []
    try:
        for r in range(nparts):
            sz = PartSizesC()
            rc = L.sfr_part_sizes_of(h, r, ctypes.byref(sz))
            if rc != 0:
                raise _sv.SolverError(rc, "sfr_part_sizes_of")
            a = dict(ia=np.zeros(sz.ia_len, np.int32), ja=np.zeros(sz.nAd + sz.nAdR, np.int32),
                     src=np.zeros(sz.nAd + sz.nAdR, np.int32), l2g=np.zeros(sz.nEq, np.int32),
                     iaSends=np.zeros(sz.nVizPart + 1, np.int32),
                     iaRcvs=np.zeros(sz.nVizPart + 1, np.int32),
                     fMap=np.zeros(sz.nRcvs + sz.nSends, np.int32),
                     vizPart=np.zeros(sz.nVizPart, np.int16))
            rc = L.sfr_part_fill(h, r, *(_sv._ptr(a[k]) for k in
                                         ("ia", "ja", "src", "l2g", "iaSends", "iaRcvs",
                                          "fMap", "vizPart")))
            if rc != 0:
                raise _sv.SolverError(rc, "sfr_part_fill")
            out.append(Layout(rank=r, unsym=bool(unsym), nEq=sz.nEq, nEqNov=sz.nEqNov,
                              nAd=sz.nAd, nAdR=sz.nAdR, **a))
    finally:
        L.sfr_part_destroy(h)
    return out


def check_layouts(layouts: list[Layout]) -> list[str]:
    """Problems in a complete set of layouts (one process): each rank must
    receive from every neighbour what that neighbour sends it, in order."""
    by_rank = {lay.rank: lay for lay in layouts}
    msgs = []
    for lay in layouts:
        for n, p in enumerate(lay.vizPart.tolist()):
            got = lay.receives_from(n)
            other = by_rank.get(p)
            if other is None:
                msgs.append(f"rank {lay.rank}: neighbour {p} missing")
                continue
            m = np.flatnonzero(other.vizPart == lay.rank)
            sent = other.sends_to(int(m[0])) if len(m) else np.zeros(0, np.int32)
            if not np.array_equal(got, sent):
                msgs.append(f"rank {lay.rank} expects {len(got)} values from rank {p}, "
                            f"which sends {len(sent)}"
                            + ("" if len(got) != len(sent) else " in another order"))
    return msgs


def check_interfaces(layout: Layout, group=None) -> list[str]:
    """The same check over a torch.distributed process group: every rank
    publishes what it sends and expects, by global equation.  Returns the
    same list of problems on every rank."""
    import torch.distributed as dist
    mine = {"rank": layout.rank,
            "viz": layout.vizPart.tolist(),
            "send": [layout.sends_to(n).tolist() for n in range(len(layout.vizPart))],
            "recv": [layout.receives_from(n).tolist() for n in range(len(layout.vizPart))]}
    world = dist.get_world_size(group)
    allv = [None] * world
    dist.all_gather_object(allv, mine, group=group)
    msgs = []
    by_rank = {d["rank"]: d for d in allv}
    if len(by_rank) != world:
        msgs.append("two processes claim the same rank")
    for d in allv:
        for n, p in enumerate(d["viz"]):
            o = by_rank.get(p)
            if o is None:
                msgs.append(f"rank {d['rank']}: neighbour {p} is not in the group")
                continue
            sent = o["send"][o["viz"].index(d["rank"])] if d["rank"] in o["viz"] else []
            if sent != d["recv"][n]:
                msgs.append(f"rank {d['rank']} expects {len(d['recv'][n])} values from "
                            f"rank {p}, which sends {len(sent)}"
                            + ("" if len(sent) != len(d["recv"][n]) else " in another order"))
    return msgs


class _Group:
    def __init__(self):
        self._h = _P()
        self.members: list["DistSystem"] = []

    def close(self):
        if self._h:
            for s in list(self.members):
                s.close()
            _lib().sfr_dist_group_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LocalGroup(_Group):
    """All ranks in this process, on one device."""

    def __init__(self, nparts: int, device: int = 0):
        super().__init__()
        self.nranks = int(nparts)
        self.device = int(device)
        rc = _lib().sfr_dist_group_local(self.nranks, self.device, ctypes.byref(self._h))
        if rc != 0:
            raise _sv.SolverError(rc, "sfr_dist_group_local")


def nccl_unique_id() -> bytes:
    buf = (ctypes.c_uint8 * 128)()
    rc = _lib().sfr_dist_nccl_id(buf)
    if rc != 0:
        raise _sv.SolverError(rc, "sfr_dist_nccl_id")
    return bytes(buf)


class NcclGroup(_Group):
    """One rank per process (torchrun), NCCL for the halo and the sums."""

    def __init__(self, nranks: int, rank: int, uid: bytes, device: int):
        super().__init__()
        self.nranks, self.rank, self.device = int(nranks), int(rank), int(device)
        if len(uid) != 128:
            raise ValueError("the NCCL id is 128 bytes")
        buf = (ctypes.c_uint8 * 128).from_buffer_copy(uid)
        rc = _lib().sfr_dist_group_nccl(self.nranks, self.rank, buf, self.device,
                                        ctypes.byref(self._h))
        if rc != 0:
            raise _sv.SolverError(rc, "sfr_dist_group_nccl")

    @classmethod
    def from_process_group(cls, device: int, group=None) -> "NcclGroup":
        """Rank 0 of the torch.distributed group makes the id; every rank
        receives it and joins."""
        import torch.distributed as dist
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        box = [nccl_unique_id() if rank == 0 else None]
        dist.broadcast_object_list(box, src=dist.get_global_rank(group, 0)
                                   if group is not None else 0, group=group)
        return cls(world, rank, box[0], device)


class DistSystem:
    """One rank's partition resident on its group's device."""

    def __init__(self, group: _Group, layout: Layout):
        self.group = group
        self.layout = layout
        self._iface = layout.interface()
        self._h = _P()
        rc = _lib().sfr_gpu_dist_create_storage(
            group._h, layout.rank, int(layout.storage), layout.nEq, layout.nEqNov, layout.nAd,
            layout.nAdR, _sv._ptr(layout.ia), _sv._ptr(layout.ja), int(layout.unsym),
            ctypes.byref(self._iface), ctypes.byref(self._h))
        if rc != 0:
            raise _sv.SolverError(rc, "sfr_gpu_dist_create_storage: " + _sv.last_error())
        group.members.append(self)

    def set_values(self, al, ad) -> None:
        al, ad = _sv._f64(al), _sv._f64(ad)
        if len(al) != value_count(self.layout) or len(ad) != self.layout.nEqNov:
            raise ValueError("al must hold the storage's values and ad nEqNov")
        rc = _lib().sfr_gpu_dist_set_values(self._h, _sv._ptr(al), _sv._ptr(ad))
        if rc != 0:
            raise _sv.SolverError(rc, "sfr_gpu_dist_set_values")

    def close(self):
        if self._h:
            _lib().sfr_gpu_dist_destroy(self._h)
            self._h = _P()
            if self in self.group.members:
                self.group.members.remove(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_solverC_group(group: "NcclGroup | None") -> None:
    """Route sfr_solverC through the MPI branch on this NCCL group (None:
    back to the single-GPU path)."""
    rc = _lib().sfr_solverC_set_group(None if group is None else group._h)
    if rc != 0:
        raise _sv.SolverError(rc, "sfr_solverC_set_group")


def solve(group: _Group, systems: list[DistSystem], solver: int, b, x0=None, tol=1e-10,
          maxit=100000, newx=True):
    """mpiPcg / mpiPbicgstab over the ranks this process holds (every rank
    of a LocalGroup in rank order, or this process's one rank).  b[r]: the
    rank's rows of b; x0[r]: its nEq entries (ghosts included) when newx is
    false.  Returns ([x_r with nEq entries], SolveInfo)."""
    k = len(systems)
    bs = [_sv._f64(v) for v in b]
    xs = []
    for r, s in enumerate(systems):
        if len(bs[r]) != s.layout.nEqNov:
            raise ValueError("b[r] must hold the rank's nEqNov rows")
        x = np.zeros(s.layout.nEq) if x0 is None else np.array(x0[r], dtype=np.float64)
        if len(x) != s.layout.nEq:
            raise ValueError("x0[r] must hold the rank's nEq entries")
        xs.append(x)
    hs = (_P * k)(*[s._h for s in systems])
    bp = (_P * k)(*[_sv._ptr(v) for v in bs])
    xp = (_P * k)(*[_sv._ptr(v) for v in xs])
    info = _sv.SolveInfoC()
    rc = _lib().sfr_gpu_dist_solve(group._h, k, hs, int(solver), bp, xp, float(tol), int(maxit),
                                   int(bool(newx)), ctypes.byref(info))
    if rc < 0:
        raise _sv.SolverError(rc, "sfr_gpu_dist_solve")
    return xs, _sv.SolveInfo.from_c(info)
