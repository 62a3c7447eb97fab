"""Slab decomposition along x across ranks (one process per GPU): which x-planes a rank
owns, and the halo exchange of one time step.

A domain of Nx planes (ghosts included, interior planes 1 .. Nx-2) is cut into `world`
slabs of consecutive interior planes; rank r's lattice holds its planes plus one halo plane
on each side (the global ghost plane where the slab touches the domain's end).  Each step:

    collide (Collide_Species + Collide) -> exchange(POPULATIONS) -> Streaming, TMS_BC,
    calculate_moment -> exchange(RECORD)

exchange() packs the face planes, sends the face-1 values to the upper neighbour and the
face-0 values to the lower one, receives the lower neighbour's face-1 values into its own
face 0 and the upper neighbour's face-0 values into face 1, and unpacks.  With a periodic x
domain the first and the last rank are neighbours.  The four point-to-point operations are
issued in one fixed order -- send up, send down, receive from down, receive from up -- so
that transports which match a pair's messages in issue order (NCCL) and transports that match
them by tag (gloo) pair them the same way, also when world == 2 and both neighbours are the
same rank.
"""

POPULATIONS, RECORD = 0, 1
TAG_UP, TAG_DOWN = 1, 0


def partition(n_interior, world, rank):
    """The global interior planes [a, b] (inclusive, 1-based as in the reference's lattice)
    rank owns: consecutive, sizes differing by at most one."""
    base, extra = divmod(n_interior, world)
    a = 1 + rank * base + min(rank, extra)
    return a, a + base + (1 if rank < extra else 0) - 1


def neighbours(world, rank, periodic=True):
    up = rank + 1 if rank + 1 < world else (0 if periodic else None)
    down = rank - 1 if rank > 0 else (world - 1 if periodic else None)
    return up, down


def exchange(what, pack, unpack, comm, world, rank, periodic=True):
    """One halo exchange.  pack(face, what) -> send buffer; unpack(face, what, buffer);
    comm.sendrecv(ops) runs [(kind, buffer, peer, tag), ...] with kind "send"/"recv" and
    returns once all have completed; comm.empty_like(buffer) makes a receive buffer."""
    up, down = neighbours(world, rank, periodic)
    to_up = pack(1, what) if up is not None else None
    to_down = pack(0, what) if down is not None else None
    from_down = comm.empty_like(to_up if to_up is not None else to_down) if down is not None else None
    from_up = comm.empty_like(to_down if to_down is not None else to_up) if up is not None else None
    ops = []
    if up is not None:
        ops.append(("send", to_up, up, TAG_UP))
    if down is not None:
        ops.append(("send", to_down, down, TAG_DOWN))
        ops.append(("recv", from_down, down, TAG_UP))
    if up is not None:
        ops.append(("recv", from_up, up, TAG_DOWN))
    comm.sendrecv(ops)
    if down is not None:
        unpack(0, what, from_down)
    if up is not None:
        unpack(1, what, from_up)


class TorchComm:
    """comm for exchange() over torch.distributed (gloo on host tensors, NCCL on device
    tensors): the operations batched into one group (batch_isend_irecv)."""

    def __init__(self, dist):
        self.dist = dist

    def empty_like(self, t):
        import torch
        return torch.empty_like(t)

    def sendrecv(self, ops):
        d = self.dist
        p2p = [d.P2POp(d.isend if kind == "send" else d.irecv, buf, peer, tag=tag) for kind, buf, peer, tag in ops]
        for req in d.batch_isend_irecv(p2p):
            req.wait()
