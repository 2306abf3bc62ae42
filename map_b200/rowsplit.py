"""One raster split over ranks by row bands (one process per GPU).

The reference's runtime has multi-device placeholders only
(runtime/Config.hpp:26 `max_num_devices`, runtime/Runtime.cpp:110-111 forces
one device); this module is the multi-GPU form of its Local / Focal path:

  * RowSplit: rank r owns rows [y0, y1) of an H-row raster (balanced bands)
    and holds them with `margin` halo rows above and below (clipped to the
    raster) in one buffer of rows [ya, yb);
  * RowSplit.exchange: before a focal program runs, each rank sends its first
    and last `margin` own rows to the neighbouring ranks, which receive them
    into the halo rows of their OWN buffers (torch.distributed point-to-point
    send / recv: NCCL between GPUs, gloo on CPU). Kernels then read local
    memory only: no kernel ever addresses another GPU's memory;
  * run_rows: evaluates rows [y0, y1) of a program on this rank's device from
    band inputs (ma_fromDeviceRows / ma_evalRows: border rules are applied in
    whole-raster coordinates, so every rank's rows equal the rows of a
    one-device evaluation);
  * iterate / engine_chunk: a program applied `steps` times (Game of Life
    generations) with a halo of k rows exchanged every k steps;
  * zone_stats_allreduce: per-zone partial count / min / max / sum of every rank
    combined into the whole raster's (count and sum by SUM, min and max as
    order-preserving integer keys by MAX), identical on every rank.

Every rank takes the same collective steps in the same order.
"""


def band_rows(H, world, rank):
    """Rows [y0, y1) of rank `rank` when H rows are split into `world` bands
    whose sizes differ by at most one row."""
    if not (0 <= rank < world) or H < world:
        raise ValueError("band_rows: %d rows cannot be split over %d ranks" % (H, world))
    return H * rank // world, H * (rank + 1) // world


class RowSplit:
    """The rows this rank owns and holds of an H x W raster split over `world` ranks."""

    def __init__(self, H, W, rank, world, margin):
        self.H, self.W, self.rank, self.world, self.margin = H, W, rank, world, int(margin)
        self.y0, self.y1 = band_rows(H, world, rank)
        for r in range(world):
            a, b = band_rows(H, world, r)
            if world > 1 and b - a < self.margin:
                raise ValueError("RowSplit: band of rank %d has %d rows, fewer than the %d-row halo" % (r, b - a, margin))
        self.ya = max(0, self.y0 - self.margin)
        self.yb = min(H, self.y1 + self.margin)

    def alloc(self, dtype, device=None):
        """A zeroed buffer for the held rows [ya, yb), rows padded to a multiple of
        128 bytes (device kernels stage tiles with TMA, which needs row pitches
        in multiples of 16 bytes); the raster's cells are buf[:, :W]."""
        import torch
        es = torch.empty((), dtype=dtype).element_size()
        wp = (self.W * es + 127) // 128 * 128 // es
        return torch.zeros((self.rows, wp), dtype=dtype, device=device)

    @property
    def rows(self):
        """Rows held (own + halo)."""
        return self.yb - self.ya

    def own(self, buf):
        """The own rows [y0, y1) of a held-rows buffer (rows [ya, yb))."""
        return buf[self.y0 - self.ya:self.y1 - self.ya]

    def exchange(self, buf, dist):
        """Fills the halo rows of `buf` (this rank's rows [ya, yb), a row-major
        tensor) from the neighbouring ranks' own rows. Tensors on a GPU are sent
        directly (NCCL); with a CPU backend (gloo) device tensors are staged
        through host memory."""
        if dist is None or self.world == 1 or self.margin == 0:
            return
        m = self.margin
        stage = buf.is_cuda and dist.get_backend() == "gloo"
        up, down = self.rank - 1, self.rank + 1
        sends, recvs = [], []
        if up >= 0:
            sends.append((buf[self.y0 - self.ya:self.y0 - self.ya + m], up))
            recvs.append((buf[0:self.y0 - self.ya], up))
        if down < self.world:
            sends.append((buf[self.y1 - self.ya - m:self.y1 - self.ya], down))
            recvs.append((buf[self.y1 - self.ya:self.yb - self.ya], down))
        reqs, landing = [], []
        for t, peer in recvs:
            dst = t.cpu() if stage else t
            reqs.append(dist.irecv(dst, src=peer))
            landing.append((t, dst))
        keep = []
        for t, peer in sends:
            src = t.cpu() if stage else t.contiguous()
            keep.append(src)
            reqs.append(dist.isend(src, dst=peer))
        for q in reqs:
            q.wait()
        for t, dst in landing:
            if dst is not t:
                t.copy_(dst)

    def gather(self, own, dist, root=0):
        """The whole raster on rank `root` (None elsewhere) from every rank's own rows."""
        import torch
        if dist is None or self.world == 1:
            return own.clone()
        src = own.cpu() if dist.get_backend() == "gloo" else own.contiguous()
        if self.rank == root:
            full = torch.empty((self.H,) + tuple(own.shape[1:]), dtype=own.dtype, device=src.device)
            for r in range(self.world):
                a, b = band_rows(self.H, self.world, r)
                if r == root:
                    full[a:b].copy_(src)
                else:
                    dist.recv(full[a:b], src=r)
            return full
        dist.send(src, dst=root)
        return None


def run_rows(M, split, build, inputs, out, bs=None):
    """Evaluates rows [y0, y1) of `build(*rasters)` on this rank's device.

    inputs: (tensor of rows [ya, yb), map data type) per input raster, device
    tensors row-major and contiguous; out: this rank's own-rows output tensor
    (rows [y0, y1)); bs: the raster's block size (the reference's block-mirror
    border rule depends on it). The band inputs must hold the program's halo,
    that is split.margin >= M.row_margin(program)."""
    import torch
    if out.is_cuda:
        torch.cuda.current_stream(out.device).synchronize()   # the engine's stream does not wait for torch's
    nodes = []
    for t, dt in inputs:
        pitch = t.stride(0) * t.element_size()
        nodes.append(M.from_device_rows(t.data_ptr(), pitch, [split.W, split.H], dt, split.ya, split.rows, bs=bs))
    prog = build(*nodes)
    need = M.row_margin(prog)
    if need > split.margin and (split.ya > 0 or split.yb < split.H):
        raise ValueError("run_rows: the program reads %d halo rows, the split holds %d" % (need, split.margin))
    M.eval_rows([prog], [(out.data_ptr(), out.stride(0) * out.element_size())], split.y0, split.y1)
    return prog


def iterate(split, state, steps, dist, run_chunk, chunk=None):
    """Applies a one-input program `steps` times to the split raster.

    state: this rank's buffer of rows [ya, yb) of the initial raster (halo rows
    need not be filled). Every round exchanges the halo (k = split.margin rows),
    then run_chunk(src, dst_own, n) computes n <= k steps of the program for
    the own rows, reading src (rows [ya, yb)) and writing dst_own (the own rows
    of the other buffer). Returns the buffer whose own rows hold the result."""
    import torch
    k = chunk or split.margin
    if k <= 0 or (split.world > 1 and k > split.margin):
        raise ValueError("iterate: %d steps per round need a halo of as many rows (the split holds %d)"
                         % (k, split.margin))
    a, b = state, torch.empty_like(state)
    done = 0
    while done < steps:
        n = min(k, steps - done)
        split.exchange(a, dist)
        run_chunk(a, split.own(b), n)
        a, b = b, a
        done += n
    return a


def engine_chunk(M, split, step, dtype, bs=None):
    """run_chunk for iterate() on this rank's device: n applications of `step`
    (a function of one raster) as one program evaluated over the own rows."""
    def run(src, dst_own, n):
        def build(x):
            for _ in range(n):
                x = step(x)
            return x
        run_rows(M, split, build, [(src, dtype)], dst_own, bs=bs)
    return run


# ---- per-zone statistics across ranks

def f32_key(x):
    """Order-preserving int32 key of float32 values (as an int64 tensor):
    a < b as floats exactly when key(a) < key(b) (NaN excluded)."""
    import torch
    i = x.contiguous().view(torch.int32).to(torch.int64)
    return torch.where(i >= 0, i, -(i & 0x7FFFFFFF) - 1)


def key_f32(k):
    """Inverse of f32_key."""
    import torch
    return torch.where(k >= 0, k, -k - 1 - 2 ** 31).to(torch.int32).view(torch.float32)


def zone_stats_allreduce(count, vmin, vmax, vsum, dist):
    """Combines every rank's per-zone partials (count int64, min / max float32,
    sum float32 or float64) into the whole raster's, on every rank. Zones a rank
    did not see carry count 0 (their min / max are ignored). count and sum are
    summed; min and max travel as order-preserving integer keys (f32_key) and
    are combined by MAX (min as MAX of the negated key), so they are exact and
    independent of the rank order. Returns (count, min, max, sum)."""
    import torch
    if dist is None:
        return count, vmin, vmax, vsum
    dev = count.device if dist.get_backend() != "gloo" else torch.device("cpu")
    c = count.to(dev, torch.int64).clone()
    seen = c > 0
    lo = torch.iinfo(torch.int64).min
    kmin = torch.where(seen, -f32_key(vmin.to(dev)), torch.full_like(c, lo))
    kmax = torch.where(seen, f32_key(vmax.to(dev)), torch.full_like(c, lo))
    s = vsum.to(dev).clone()
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    dist.all_reduce(kmin, op=dist.ReduceOp.MAX)
    dist.all_reduce(kmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    out_dev = count.device
    return c.to(out_dev), key_f32(-kmin).to(out_dev), key_f32(kmax).to(out_dev), s.to(out_dev)


# ---- whole-raster reductions across ranks (the zonal skeleton's D0 results)

SUM, PROD, AND, OR, MAX, MIN = 1, 2, 3, 4, 6, 7   # the map module's reduction codes (python/map.py:85)


def f64_key(x):
    """Order-preserving int64 key of float64 values: a < b as floats exactly
    when key(a) < key(b) (-0 below +0; NaN excluded)."""
    import torch
    i = x.contiguous().view(torch.int64)
    return torch.where(i >= 0, i, -(i & 0x7FFFFFFFFFFFFFFF) - 1)


def key_f64(k):
    """Inverse of f64_key."""
    import torch
    lo = torch.iinfo(torch.int64).min
    return torch.where(k >= 0, k, (-k - 1) | lo).view(torch.float64)


def zonal_allreduce(value, red, dist, bits=None, signed=True):
    """Combines every rank's reduction of its own rows (a Python number, such
    as M.value(M.zsum(band)) over the rank's own rows) into the whole raster's,
    on every rank; `red` is the map module's reduction code (zsum SUM, zprod
    PROD, zmax MAX, zmin MIN, rAND, rOR). Integers combine exactly in int64
    (wrapped to a `bits`-wide signed or unsigned type when given, as the
    raster type's arithmetic wraps);
    float sums and products combine in float64, so they agree with a
    one-device evaluation to that type's rounding; float MAX and MIN travel as
    order-preserving integer keys and are exact and independent of the rank
    order; rAND / rOR are the MIN / MAX of the ranks' truth values."""
    import numbers
    import torch
    if dist is None:
        return value
    integer = isinstance(value, numbers.Integral)       # Python or NumPy integers (bool included)
    if red in (AND, OR):
        t = torch.tensor([1 if value else 0], dtype=torch.int64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN if red == AND else dist.ReduceOp.MAX)
        return bool(t.item())
    if red in (MAX, MIN):
        if integer:
            t = torch.tensor([int(value)], dtype=torch.int64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX if red == MAX else dist.ReduceOp.MIN)
            return int(t.item())
        k = f64_key(torch.tensor([float(value)], dtype=torch.float64))
        if red == MIN:
            k = -k
        dist.all_reduce(k, op=dist.ReduceOp.MAX)
        return float(key_f64(k if red == MAX else -k).item())
    if red not in (SUM, PROD):
        raise ValueError("zonal_allreduce: unknown reduction %r" % (red,))
    op = dist.ReduceOp.SUM if red == SUM else dist.ReduceOp.PRODUCT
    if integer:
        t = torch.tensor([int(value)], dtype=torch.int64)
        dist.all_reduce(t, op=op)
        v = int(t.item())
        if bits:
            v &= (1 << bits) - 1
            if signed and v >= 1 << (bits - 1):
                v -= 1 << bits
        return v
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=op)
    return float(t.item())
