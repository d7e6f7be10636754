"""A periodic domain decomposed over ranks: each rank steps one subdomain of
the solvent and exchanges its migration and halo bags with its 26
neighbours (src/distr/flu, src/exch/flu, src/comm of the reference).

- ``Cart``: the periodic 3-D cart (MPI_Cart_create with periods, row-major
  ranks as MPI orders them) and every rank's 26 neighbours
  (comm_ini's ``ranks[i]``, src/comm/imp/ini.h).
- ``SubDomain``: one rank's subdomain on its GPU (``ctc_sub_*`` of
  libctc_b200.so): the bags are device memory, packed and unpacked by the
  library's kernels.
- ``DistTransport``: moves bags between processes with ``torch.distributed``
  point-to-point calls -- NCCL for device bags (over NVLink / NVSwitch), gloo
  for host bags.  NCCL matches the messages between two ranks in the order
  they are posted, so every rank posts its sends to a peer in the order of
  the sender's bag index and its receives from a peer in the order of the
  sender's bag index too (the receiver's bag j came from the sender's bag
  anti(j)); the tags carry the same index where the backend uses them.
- ``LocalTransport``: the ranks of one process (emulated ranks on one
  device): bag copies.
- ``step(subs, transport)``: one step of every local rank in the reference's
  order -- migrate, cell lists, pack the halo, bulk forces while the halo bags
  travel, halo forces and update.

A bag count that exceeds its capacity raises on the rank that sees it; the
other ranks then wait in their next exchange until the process group's
timeout ends it (the reference aborts the MPI job instead).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import CTC_RNG_REFERENCE, check, lib

FRAG_DIRS = tuple(((i + 2) % 3 - 1, (i // 3 + 2) % 3 - 1, (i // 9 + 2) % 3 - 1) for i in range(26))


def frag_d2i(d):
    """Fragment id of direction d (src/frag/dev.h:19-21)."""
    return ((d[0] + 2) % 3) + 3 * ((d[1] + 2) % 3) + 9 * ((d[2] + 2) % 3)


def frag_anti(i):
    d = FRAG_DIRS[i]
    return frag_d2i((-d[0], -d[1], -d[2]))


class Cart:
    """Periodic cart of dims[0] x dims[1] x dims[2] ranks, rank = (x dims[1] +
    y) dims[2] + z as MPI_Cart_create numbers them."""

    def __init__(self, dims):
        self.dims = tuple(int(d) for d in dims)
        if len(self.dims) != 3 or min(self.dims) < 1:
            raise ValueError("dims must be three positive ints")
        self.size = self.dims[0] * self.dims[1] * self.dims[2]

    def coords(self, rank):
        d = self.dims
        return (rank // (d[1] * d[2]), (rank // d[2]) % d[1], rank % d[2])

    def rank(self, coords):
        d = self.dims
        c = [int(coords[k]) % d[k] for k in range(3)]
        return (c[0] * d[1] + c[1]) * d[2] + c[2]

    def neighbours(self, rank):
        """The rank in each of the 26 directions (periodic)."""
        c = self.coords(rank)
        return [self.rank([c[k] + FRAG_DIRS[f][k] for k in range(3)]) for f in range(26)]

    def origin(self, rank, L):
        """Global coordinate of the centre of rank's subdomain of edge L, in a
        domain [0, dims * L) per axis."""
        c = self.coords(rank)
        return tuple((c[k] + 0.5) * L[k] for k in range(3))


def _view(addr, n, dtype, device):
    """A tensor over n elements of device memory at addr (no copy)."""
    import torch
    if n <= 0:
        return torch.empty(0, dtype=dtype, device=device)
    typestr = {torch.int32: "<i4", torch.float32: "<f4"}[dtype]

    class _Dev:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (addr, False), "version": 2}

    return torch.as_tensor(_Dev(), device=device)


class SubDomain:
    """One rank's subdomain (``ctc_sub``): box L in cells centred on its own
    origin, the rank's place in ``cart``, solvent DPD parameters ``dpd``."""

    REC = 8          # floats per exchanged record (two float4)

    def __init__(self, L, cart, rank, maxp, dpd, mass=1.0, dt=5e-4, bodyf=(0.0, 0.0, 0.0), rng=CTC_RNG_REFERENCE,
                 maxd=20.0, device=None):
        import torch
        self.L = tuple(int(x) for x in L)
        self.cart, self.rank = cart, int(rank)
        self.nbr = cart.neighbours(self.rank)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        cfg = _lib.SubConfig()
        s = cfg.sim
        s.LX, s.LY, s.LZ = self.L
        s.maxp = int(maxp)
        s.dpd = dpd
        s.mass, s.dt = float(mass), float(dt)
        s.bodyf = (C.c_float * 3)(*bodyf)
        s.rng = int(rng)
        cfg.dims = (C.c_int * 3)(*cart.dims)
        cfg.coords = (C.c_int * 3)(*cart.coords(self.rank))
        cfg.rank = self.rank
        cfg.nbr = (C.c_int * 26)(*self.nbr)
        cfg.maxd = float(maxd)
        self.h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(lib().ctc_sub_create(C.byref(cfg), C.byref(self.h)))
        # the bag buffers as tensors, once: a fresh object has every send bag
        # at its buffer's start, and the receive bags lie at fixed offsets
        # (the prefix of the capacities); the send bags of a pack follow one
        # another in direction order (the prefix of the counts)
        self._base = []
        for kind in range(3):
            send, recv, cap = (C.c_void_p * 26)(), (C.c_void_p * 26)(), (C.c_int * 26)()
            check(lib().ctc_sub_bags(self.h, kind, send, recv, cap))
            cap = list(cap)
            el, dt = (1, torch.int32) if kind == 2 else (self.REC, torch.float32)
            tot = el * sum(cap)
            sb = _view(send[0], tot, dt, self.device)
            rb = _view(recv[0], tot, dt, self.device)
            roff = np.concatenate([[0], np.cumsum(cap)]) * el
            if kind == 2:       # the fragment-cell starts: fixed bags in both buffers
                self._fss = ([sb[roff[f]:roff[f + 1]] for f in range(26)],
                             [rb[roff[f]:roff[f + 1]] for f in range(26)], cap)
            self._base.append((sb, [rb[roff[f]:roff[f + 1]] for f in range(26)], cap))
        # the same bags as device addresses (bag_ptrs): send buffer start,
        # receive bag addresses, capacities, bytes per counted unit
        self._ptrs = {}
        for kind in range(3):
            sb, recv, cap = self._base[kind]
            unit = 4 if kind == 2 else 4 * self.REC
            rp = [r.data_ptr() for r in recv]
            sp = [b.data_ptr() for b in self._fss[0]] if kind == 2 else sb.data_ptr()
            self._ptrs[kind] = (sp, rp, list(cap), unit)

    def close(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_sub_destroy(self.h)
            self.h = None

    __del__ = close

    def _stream(self):
        import torch
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def set_solvent(self, pp, ids=None):
        """pp (n, 6) in subdomain coordinates, ids (n,) global ids (default 0..n-1)."""
        pp = np.ascontiguousarray(pp, np.float32).reshape(-1, 6)
        idp = None
        if ids is not None:
            ids = np.ascontiguousarray(ids, np.int32)
            idp = ids.ctypes.data_as(C.c_void_p)
        check(lib().ctc_sub_set_solvent(self.h, len(pp), pp.ctypes.data_as(C.c_void_p), idp, 1, self._stream()))

    def count(self):
        n = C.c_int()
        check(lib().ctc_sub_count(self.h, C.byref(n), self._stream()))
        return n.value

    def get_solvent(self):
        """(pp (n, 6) in subdomain coordinates, ids (n,)), cell-sorted [host]."""
        import torch
        n = self.count()
        pos, vel = C.c_void_p(), C.c_void_p()
        check(lib().ctc_sub_state(self.h, C.byref(pos), C.byref(vel), None, None))
        p = _view(pos.value, 4 * n, torch.float32, self.device).view(-1, 4).cpu().numpy()
        v = _view(vel.value, 4 * n, torch.float32, self.device).view(-1, 4).cpu().numpy()
        ids = p[:, 3].copy().view(np.int32)
        return np.concatenate([p[:, :3], v[:, :3]], axis=1), ids

    # -- membranes ---------------------------------------------------------------
    def set_membranes(self, pv, cell_ids, tri, nv, params, fsi, maxc, mass=0.5):
        """Cells of one template in this subdomain: pv (nc*nv, 6) in subdomain
        coordinates, cell_ids (nc,) their global ids, tri (nt, 3), room for
        maxc cells; params a dict of RbcParams fields, fsi a DpdParams."""
        import torch
        pv = np.ascontiguousarray(pv, np.float32).reshape(-1, 6)
        tri = np.ascontiguousarray(tri, np.int32).reshape(-1, 3)
        cell_ids = np.ascontiguousarray(cell_ids, np.int32)
        self.mnv = int(nv)
        with torch.cuda.device(self.device):
            check(lib().ctc_sub_set_membranes(self.h, len(cell_ids), self.mnv, len(tri), tri.ctypes.data_as(C.c_void_p),
                                              pv.ctypes.data_as(C.c_void_p), cell_ids.ctypes.data_as(C.c_void_p),
                                              int(maxc), C.byref(_lib.RbcParams(**params)), C.byref(fsi),
                                              float(mass)))
        self.maxc = int(maxc)
        self._mbase = {}
        for kind in (3, 4, 5):
            send, recv, cap = (C.c_void_p * 26)(), (C.c_void_p * 26)(), (C.c_int * 26)()
            check(lib().ctc_sub_bags(self.h, kind, send, recv, cap))
            cap = list(cap)
            el = {3: self.REC * self.mnv, 4: self.REC, 5: 4}[kind]
            tot = el * sum(cap)
            # the cells leaving in one step fit the maxc cells' send buffer
            stot = el * self.maxc if kind == 3 else tot
            self._mbase[kind] = (_view(send[0], stot, torch.float32, self.device),
                                 _view(recv[0], tot, torch.float32, self.device), cap, el)
            rp = [recv[0] + 4 * el * cap[0] * f for f in range(26)] if kind != 5 else recv[0]
            self._ptrs[kind] = (send[0], rp, cap, 4 * el)

    def membrane_forces(self):
        """The last step's vertex forces (nc*nv, 3) and their global vertex ids [host]."""
        import torch
        nc, nv = C.c_int(), C.c_int()
        check(lib().ctc_sub_get_membranes(self.h, C.byref(nc), C.byref(nv), None, None, self._stream()))
        n = nc.value * nv.value
        pos, frc = C.c_void_p(), C.c_void_p()
        check(lib().ctc_sub_membrane_state(self.h, C.byref(pos), None, C.byref(frc)))
        torch.cuda.synchronize(self.device)
        p = _view(pos.value, 4 * n, torch.float32, self.device).view(-1, 4).cpu().numpy()
        f = _view(frc.value, 4 * n, torch.float32, self.device).view(-1, 4).cpu().numpy()
        return f[:, :3], p[:, 3].copy().view(np.int32)

    def has_membranes(self):
        return bool(getattr(self, "mnv", 0))

    def get_membranes(self):
        """(pv (nc*nv, 6) in subdomain coordinates, cell ids (nc,)) [host]."""
        nc, nv = C.c_int(), C.c_int()
        check(lib().ctc_sub_get_membranes(self.h, C.byref(nc), C.byref(nv), None, None, self._stream()))
        pv = np.zeros((nc.value * nv.value, 6), np.float32)
        ids = np.zeros(nc.value, np.int32)
        if nc.value:
            check(lib().ctc_sub_get_membranes(self.h, None, None, pv.ctypes.data_as(C.c_void_p),
                                              ids.ctypes.data_as(C.c_void_p), self._stream()))
        return pv, ids

    def mem_bags(self, kind, counts, rcounts=None):
        """Send bags (sized by counts) and receive bags of membrane kind 3
        (cells), 4 (images) or 5 (the images' forces sent back: send bag j
        holds rcounts[j] of the images received from direction j, receive
        bag f the forces on this rank's image bag f of counts[f] images)."""
        sb, rb, cap, el = self._mbase[kind]
        send, recv = [], []
        if kind == 5:
            o = 0
            for j in range(26):
                send.append(sb[o:o + el * rcounts[j]])
                o += el * rcounts[j]
            o = 0
            for f in range(26):
                recv.append(rb[o:o + el * counts[f]])
                o += el * counts[f]
            return send, recv, cap
        o = 0
        for f in range(26):
            send.append(sb[o:o + el * counts[f]])
            o += el * counts[f]
        recv = [rb[el * cap[0] * f:el * cap[0] * (f + 1)] for f in range(26)]
        return send, recv, cap

    def mem_distr_pack(self):
        check(lib().ctc_sub_mem_distr_pack(self.h, self._stream()))

    def mem_distr_counts(self):
        c = (C.c_int * 26)()
        check(lib().ctc_sub_mem_distr_counts(self.h, c))
        return list(c)

    def mem_distr_unpack(self, rcounts):
        check(lib().ctc_sub_mem_distr_unpack(self.h, (C.c_int * 26)(*rcounts), self._stream()))

    def mem_exch_pack(self):
        check(lib().ctc_sub_mem_exch_pack(self.h, self._stream()))

    def mem_exch_counts(self):
        c = (C.c_int * 26)()
        check(lib().ctc_sub_mem_exch_counts(self.h, c))
        return list(c)

    def mem_fsi(self, rcounts):
        check(lib().ctc_sub_mem_fsi(self.h, (C.c_int * 26)(*rcounts), self._stream()))

    def mem_update(self):
        check(lib().ctc_sub_mem_update(self.h, self._stream()))

    def forces(self):
        """The last step's forces (n, 3), cell-sorted [host]."""
        import torch
        n = self.count()
        f = C.c_void_p()
        check(lib().ctc_sub_state(self.h, None, None, C.byref(f), None))
        return _view(f.value, 4 * n, torch.float32, self.device).view(-1, 4)[:, :3].cpu().numpy()

    def seeds(self):
        out = (C.c_float * 27)()
        check(lib().ctc_sub_seeds(self.h, out))
        return np.array(out, np.float32)

    def bags(self, kind, counts):
        """Device tensors of the send bags (their counts, as the last pack
        left them) and the receive bags (full capacity) of kind 0
        (migration), 1 (halo records) or 2 (halo fragment-cell starts)."""
        if kind == 2:
            return self._fss
        sb, recv, cap = self._base[kind]
        send, o = [], 0
        for f in range(26):
            e = o + self.REC * counts[f]
            send.append(sb[o:e])
            o = e
        return send, recv, cap

    def bag_ptrs(self, kind, counts, rcounts=None):
        """The bags of bags() (kinds 0-2) and mem_bags() (kinds 3-5) as device
        addresses, for a transport whose ranks share a process: (send
        addresses, the units each sends, receive addresses, their capacities
        in units, bytes per unit).  Kind 2 sends its fixed bags whole; kind 5
        sends rcounts[j] forces from bag j and receives counts[f] into bag f."""
        sp, rp, cap, unit = self._ptrs[kind]
        if kind == 2:
            return sp, cap, rp, cap, unit
        sent = rcounts if kind == 5 else counts
        send, o = [], sp
        for f in range(26):
            send.append(o)
            o += unit * sent[f]
        if kind == 5:
            recv, o = [], rp
            for f in range(26):
                recv.append(o)
                o += unit * counts[f]
            return send, sent, recv, counts, unit
        return send, sent, rp, cap, unit

    # -- the phases of a step ------------------------------------------------
    def distr_pack(self):
        check(lib().ctc_sub_distr_pack(self.h, self._stream()))

    def distr_counts(self):
        c = (C.c_int * 26)()
        check(lib().ctc_sub_distr_counts(self.h, c))
        return list(c)

    def distr_unpack(self, rcounts):
        check(lib().ctc_sub_distr_unpack(self.h, (C.c_int * 26)(*rcounts), self._stream()))

    def exch_pack(self):
        check(lib().ctc_sub_exch_pack(self.h, self._stream()))

    def exch_counts(self):
        c = (C.c_int * 26)()
        check(lib().ctc_sub_exch_counts(self.h, c))
        return list(c)

    def bulk(self):
        check(lib().ctc_sub_bulk(self.h, self._stream()))

    def halo_update(self, rcounts):
        check(lib().ctc_sub_halo_update(self.h, (C.c_int * 26)(*rcounts), self._stream()))


def _counts_tensor(counts, device):
    import torch
    return torch.tensor(counts, dtype=torch.int32, device=device)


class LocalTransport:
    """All ranks of the cart in this process (``subs[r]`` is rank r):
    the bag of rank r for direction f goes to bag anti(f) of rank nbr_r[f]."""

    def __init__(self, cart):
        self.cart = cart
        self.nbr = [cart.neighbours(r) for r in range(cart.size)]
        self.anti = [frag_anti(f) for f in range(26)]

    def exchange_counts(self, counts):
        """counts[r][f] sent by rank r in direction f -> received [r][j]."""
        out = [[0] * 26 for _ in counts]
        anti = self.anti
        for r, c in enumerate(counts):
            nbr = self.nbr[r]
            for f in range(26):
                out[nbr[f]][anti[f]] = c[f]
        return out

    def exchange_ptrs(self, bags, stream):
        """bags[r] = SubDomain.bag_ptrs(...) of rank r: every send bag copied
        into its receive bag with one launch (ctc_bags_copy) on stream."""
        src, dst, nbytes = [], [], []
        anti = self.anti
        for r, (sp, sent, _, _, unit) in enumerate(bags):
            nbr = self.nbr[r]
            for f in range(26):
                if sent[f]:
                    q, j = nbr[f], anti[f]
                    if sent[f] > bags[q][3][j]:
                        raise ValueError("bag %d of rank %d: %d units into %d" % (f, r, sent[f], bags[q][3][j]))
                    src.append(sp[f])
                    dst.append(bags[q][2][j])
                    nbytes.append(sent[f] * unit)
        if src:
            k = len(src)
            check(lib().ctc_bags_copy(k, (C.c_void_p * k)(*dst), (C.c_void_p * k)(*src),
                                      (C.c_longlong * k)(*nbytes), stream))
        return _Done()

    def exchange(self, sends, recvs, rcounts, rec):
        """sends[r][f] (sized), recvs[r][j] (capacity) tensors; rcounts[r][j]
        the elements / rec received in bag j of rank r.  Device bags move in
        one launch (ctc_bags_copy) on the current stream; the handle's wait()
        is a no-op."""
        src, dst, nbytes = [], [], []
        dev = None
        for r, s in enumerate(sends):
            nbr = self.cart.neighbours(r)
            for f in range(26):
                n = s[f].numel()
                if not n:
                    continue
                d = recvs[nbr[f]][frag_anti(f)]
                if n > d.numel() or d.dtype != s[f].dtype:
                    raise ValueError("bag %d of rank %d: %d elements into %d" % (f, r, n, d.numel()))
                if s[f].is_cuda:
                    dev = s[f].device
                    src.append(s[f].data_ptr())
                    dst.append(d.data_ptr())
                    nbytes.append(n * s[f].element_size())
                else:
                    d[:n].copy_(s[f])
        if src:
            import torch
            k = len(src)
            check(lib().ctc_bags_copy(k, (C.c_void_p * k)(*dst), (C.c_void_p * k)(*src),
                                      (C.c_longlong * k)(*nbytes),
                                      C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
        return _Done()


class _Done:
    def wait(self):
        pass


class _Posted:
    def __init__(self, works):
        self.works = works

    def wait(self):
        for w in self.works:
            w.wait()
        self.works = []


class DistTransport:
    """This process is rank ``rank`` of ``group`` (default: the world); bags
    move with torch.distributed point-to-point calls."""

    def __init__(self, cart, rank, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.cart, self.rank, self.group = cart, int(rank), group
        self.nbr = cart.neighbours(self.rank)
        self.dist = dist
        self.device = device if device is not None else torch.device("cpu")
        if dist.get_world_size(group) != cart.size:
            raise ValueError("the cart has %d ranks, the group %d" % (cart.size, dist.get_world_size(group)))

    def _global(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def _post(self, sends, recvs):
        """sends[f] to nbr[f] (bag f), recvs[j] from nbr[j] (the sender's bag
        anti(j)); self-messages are copies.  Returns a handle whose wait()
        makes the current stream (NCCL) or the host (gloo) wait for all."""
        dist = self.dist
        ops = []
        for f in range(26):
            if self.nbr[f] == self.rank:
                if sends[f] is not None and sends[f].numel():
                    recvs[frag_anti(f)][:sends[f].numel()].copy_(sends[f])
                continue
            if sends[f] is not None and sends[f].numel():
                ops.append((self.nbr[f], f, "s", sends[f]))
        for j in range(26):
            if self.nbr[j] == self.rank or recvs[j] is None or not recvs[j].numel():
                continue
            ops.append((self.nbr[j], frag_anti(j), "r", recvs[j]))
        # per peer, in the order of the sender's bag index; sends and receives
        # interleaved in one batch so that no pair of ranks waits on the other
        ops.sort(key=lambda o: (o[0], o[1], o[2]))
        p2p = []
        for peer, tag, kind, t in ops:
            fn = dist.isend if kind == "s" else dist.irecv
            p2p.append(dist.P2POp(fn, t, self._global(peer), self.group, tag))
        return _Posted(dist.batch_isend_irecv(p2p) if p2p else [])

    def exchange_counts(self, counts):
        import torch
        c = counts[0]
        send = torch.tensor(c, dtype=torch.int32, device=self.device)
        recv = torch.zeros(26, dtype=torch.int32, device=self.device)
        self._post([send[f:f + 1] for f in range(26)], [recv[j:j + 1] for j in range(26)]).wait()
        return [recv.cpu().tolist()]

    def exchange(self, sends, recvs, rcounts, rec):
        """Posts this rank's bags (sends[0], recvs[0], rcounts[0]); returns the
        handle to wait on."""
        s, r, rc = sends[0], recvs[0], rcounts[0]
        return self._post(s, [r[j][:rec * rc[j]] for j in range(26)])


def step(subs, transport, marks=None):
    """One step of every rank in ``subs`` (one SubDomain per local rank, in
    rank order for a LocalTransport, just this rank's for a DistTransport):
    distribute_flu, the cell lists, forces (bulk while the halo bags
    travel, then the halo) and the update -- src/sim/imp/run.h:8-68 for
    the solvent.  marks (a list) receives a CUDA event recorded on the
    current stream after the migration, after the cell lists, after the halo
    exchange and at the end."""
    def mark():
        if marks is not None:
            import torch
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            marks.append(e)
    R = SubDomain.REC
    mem = bool(getattr(subs[0], "mnv", 0))
    direct = hasattr(transport, "exchange_ptrs")    # ranks of one process: bags by address

    def move(kind, counts, rcounts, rec, back=None):
        """Bags of one kind from every rank to its neighbours; counts the send
        sizes (kind 5: the forces go back for the images rcounts came from)."""
        if direct:
            if kind == 5:
                ptrs = [s.bag_ptrs(5, c, b) for s, c, b in zip(subs, counts, back)]
            elif kind == 2:
                ptrs = [s.bag_ptrs(2, None) for s in subs]
            else:
                ptrs = [s.bag_ptrs(kind, c) for s, c in zip(subs, counts)]
            return transport.exchange_ptrs(ptrs, subs[0]._stream())
        if kind == 2:
            bags = [s.bags(2, None) for s in subs]
            return transport.exchange([b[0] for b in bags], [b[1] for b in bags], [b[2] for b in bags], rec)
        if kind == 5:
            bags = [s.mem_bags(5, c, b) for s, c, b in zip(subs, counts, back)]
        else:
            bags = [(s.bags if kind < 3 else s.mem_bags)(kind, c) for s, c in zip(subs, counts)]
        return transport.exchange([b[0] for b in bags], [b[1] for b in bags], rcounts, rec)

    for s in subs:
        s.distr_pack()
        if mem:     # whole cells migrate beside the solvent (distr_rbc)
            s.mem_distr_pack()
    counts = [s.distr_counts() for s in subs]
    rcounts = transport.exchange_counts(counts)
    move(0, counts, rcounts, R).wait()
    if mem:
        ccounts = [s.mem_distr_counts() for s in subs]
        crc = transport.exchange_counts(ccounts)
        move(3, ccounts, crc, R * subs[0].mnv).wait()
        for s, rc in zip(subs, crc):
            s.mem_distr_unpack(rc)
    mark()
    for s, rc in zip(subs, rcounts):
        s.distr_unpack(rc)
    mark()
    for s in subs:
        s.exch_pack()
        if mem:     # the vertices' images for the neighbours' FSI (exch_obj)
            s.mem_exch_pack()
    # the bulk forces run on each subdomain's own stream while the host
    # collects the halo counts and the halo bags travel
    for s in subs:
        s.bulk()
    counts = [s.exch_counts() for s in subs]
    rcounts = transport.exchange_counts(counts)
    h1 = move(1, counts, rcounts, R)
    h2 = move(2, None, None, 1)
    if mem:
        icounts = [s.mem_exch_counts() for s in subs]
        irc = transport.exchange_counts(icounts)
        move(4, icounts, irc, R).wait()
    h1.wait()
    h2.wait()
    if mem:     # FSI of the own vertices and of the images; the images' forces go back
        for s, rc in zip(subs, irc):
            s.mem_fsi(rc)
        move(5, icounts, icounts, 4, back=irc).wait()
    mark()
    for s, rc in zip(subs, rcounts):
        s.halo_update(rc)
    if mem:
        for s in subs:
            s.mem_update()
    mark()
