"""Channel-partitioned multi-GPU layout: every rank beamforms its own block
of channels (no exchange), then one all-to-all turns the per-rank channel
blocks of the coherent beams into per-rank beam blocks with every channel,
which is what incoherent dedispersion needs (it sums over all channels of a
beam).  NCCL on GPUs (device tensors), gloo on CPU; no TMA or multicast.

The reference scales out with one process per frequency bridge and runs its
incoherent dedisperser per bridge (cpp/skyweaver/MultiBeamWriter.hpp:18-40,
detail/IncoherentDedispersionPipeline.cu:6-113); the exchange lets one
dedisperser see the whole band.
"""
from __future__ import annotations


def rank_channels(nchans_total: int, world: int, rank: int) -> slice:
    """The contiguous channel block of `rank` (equal blocks)."""
    if nchans_total % world:
        raise ValueError(f"{nchans_total} channels do not split over {world} ranks")
    n = nchans_total // world
    return slice(rank * n, (rank + 1) * n)


def rank_beams(nbeams: int, world: int, rank: int) -> slice:
    """The contiguous beam block that `rank` dedisperses after the exchange."""
    if nbeams % world:
        raise ValueError(f"{nbeams} beams do not split over {world} ranks")
    n = nbeams // world
    return slice(rank * n, (rank + 1) * n)


def channels_to_beams(tfb, group=None):
    """All-to-all of coherent beams: this rank's TFB [T][F_local][B] (channels
    of its block, every beam) -> [T][world * F_local][B / world] (every
    channel, in rank order, of this rank's beam block).  One collective;
    tensors stay on their device."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    T, F, B = tfb.shape[:3]
    rest = tuple(tfb.shape[3:])
    if B % world:
        raise ValueError(f"{B} beams do not split over {world} ranks")
    send = tfb.reshape(T, F, world, B // world, *rest).movedim(2, 0).contiguous()
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    # recv[src] = [T][F_local][B / world] of the source rank's channel block
    return recv.movedim(0, 1).reshape(T, world * F, B // world, *rest)


class ChannelChain:
    """One rank's part of the channel-partitioned chain:

        beamform this rank's channel block  ->  channels_to_beams (one
        all-to-all)  ->  incoherent dedispersion of this rank's beam block
        over every channel

    `beamform(voltages)` returns the coherent beams of the rank's channels,
    TFB [T][F_local][B] (e.g. a BeamformerPipeline's device output);
    `dedisperse(tfb)` takes [T][F_total][B / world] and returns the rank's
    dedispersed beams (e.g. stages.incoherent_dedisperse with the whole
    band's delays, or an IncoherentDedispersionPipeline push).  The stages
    stay on the rank's device; the only collective is the exchange.  The
    reference instead runs one process per bridge and dedisperses each
    bridge on its own channels (MultiBeamWriter.hpp:18-40,
    detail/IncoherentDedispersionPipeline.cu:6-113)."""

    def __init__(self, beamform, dedisperse, group=None):
        self.beamform = beamform
        self.dedisperse = dedisperse
        self.group = group

    def __call__(self, voltages):
        tfb = self.beamform(voltages)
        return self.dedisperse(channels_to_beams(tfb, self.group))
