"""Chunked sequence decode, and its sharding over ranks (one process per GPU).

The decoder stage exports a sequence in chunks of `chunk_frames` frames,
each decoded as one DecodeFrameSequenceWindow call over the chunk plus
`chunk_overlap` frames of temporal context on each side, clipped to the
sequence (hvd_chroma_decoder_stage.cpp:986-1060 drives the chunks,
:706-735 builds each window; hvd_config.h:392-404). The context frames are
decoded inside the window but only the chunk's own frames are kept, so the
chunks are independent: every chunk reads its halo frames itself and no
chunk waits for another. With the temporal terms off (temporal_strength < 0
or no CG iterations) the fields are decoupled and the overlap is 0.

Across GPUs the chunks are therefore shared out with no collective on the
data path: rank r decodes chunks r, r + world, r + 2 world, ... (the halo
frames of a chunk are read by whichever rank decodes it), and the decoded
frames are gathered in chunk order only where one process must write them
(`gather_frames`, over torch.distributed).
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Chunk:
    index: int         # chunk number in sequence order
    first: int         # first core frame (sequence frame id)
    last: int          # last core frame (inclusive)
    w0: int            # first frame of the window (core minus the leading overlap)
    w1: int            # last frame of the window (inclusive)

    @property
    def core_begin(self) -> int:
        """Index of the first core frame inside the window."""
        return self.first - self.w0

    @property
    def core_end(self) -> int:
        """One past the last core frame inside the window."""
        return self.last - self.w0 + 1


def plan_chunks(first: int, last: int, chunk_frames: int = 6, chunk_overlap: int = 1,
                coupled: bool = True) -> list[Chunk]:
    """The stage's export chunks over frames [first, last]: cores of
    max(1, chunk_frames) frames; windows extended by chunk_overlap frames
    each side when the temporal terms couple the fields, clipped to the
    sequence (hvd_chroma_decoder_stage.cpp:711-716, 997-1060)."""
    if last < first:
        return []
    step = max(1, int(chunk_frames))
    ov = max(0, int(chunk_overlap)) if coupled else 0
    out = []
    t0 = first
    while t0 <= last:
        t1 = min(t0 + step - 1, last)
        w0 = t0 - ov if t0 > first + ov else first
        w1 = min(t1 + ov, last)
        out.append(Chunk(len(out), t0, t1, w0, w1))
        t0 = t1 + 1
    return out


def is_coupled(cfg) -> bool:
    """Whether the window's fields are coupled by temporal terms (the stage's
    `enable_temporal && cg_iterations > 0`, with 3-D off expressed as a
    negative temporal strength)."""
    return cfg.temporal_strength >= 0.0 and cfg.cg_iterations > 0


def shard(chunks: list[Chunk], world: int, rank: int) -> list[Chunk]:
    """The chunks rank `rank` of `world` decodes: every world-th chunk,
    starting at its rank (round robin keeps the ranks' loads within one
    chunk of each other)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    return chunks[rank::world]


def decode_chunks(decode_window, frames, chunks: list[Chunk]) -> dict[int, list]:
    """Decode each chunk's window with `decode_window(window_frames,
    core_begin, core_end)` (e.g. a bound Context.decode_frame_sequence_window)
    and keep its core frames: {chunk index: [frame, ...]}."""
    out = {}
    for c in chunks:
        got = decode_window(frames[c.w0:c.w1 + 1], c.core_begin, c.core_end)
        if len(got) != c.core_end - c.core_begin:
            raise RuntimeError(f"chunk {c.index}: {len(got)} frames decoded, "
                               f"{c.core_end - c.core_begin} expected")
        out[c.index] = list(got)
    return out


def gather_frames(local: dict[int, list], n_chunks: int, dist=None, dst: int = 0):
    """The decoded frames of every rank, in sequence order, on rank `dst`
    (None elsewhere); without a process group, `local` must hold every
    chunk. Host objects travel through gather_object (the frames are host
    planes; the decode itself moved no data between ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        parts = [local]
    else:
        parts = [None] * dist.get_world_size() if dist.get_rank() == dst else None
        dist.gather_object(local, parts, dst=dst)
        if dist.get_rank() != dst:
            return None
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"chunk {k} decoded twice")
            merged[k] = v
    missing = [k for k in range(n_chunks) if k not in merged]
    if missing:
        raise RuntimeError(f"chunks never decoded: {missing}")
    return [fr for k in range(n_chunks) for fr in merged[k]]
