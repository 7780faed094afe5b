"""Host logic of SurfaceSampler's choice between the one-launch sample (he_sample_record)
and the three launches he_flux -> he_surface_contract -> he_volkov_add: a surface beyond the
one-launch limits (HE_ERR_SHAPE from he_sample_create) falls back to the three launches,
any other failure is raised; an engine whose surface is not this package's SurfaceFlux keeps
the three launches.  No GPU: the handle construction is replaced."""
import pytest


def test_sampler_falls_back_to_three_launches_beyond_the_one_launch_limits(monkeypatch):
    from laqphysics_b200 import streaming_surface as ss
    from laqphysics_b200._lib import HE_ERR_CUDA, HE_ERR_SHAPE, HeliumError

    def too_large(*args):
        raise HeliumError(HE_ERR_SHAPE, 'more than 16 surface rows')

    from laqphysics_b200.surface import SurfaceFlux

    class Engine:   # an engine whose surface is this package's SurfaceFlux
        surface = SurfaceFlux.__new__(SurfaceFlux)

    monkeypatch.setattr(ss, 'FusedSample', too_large)
    sampler = ss.SurfaceSampler(Engine(), object(), object())
    assert sampler.fused is None

    def broken(*args):
        raise HeliumError(HE_ERR_CUDA, 'out of memory')

    monkeypatch.setattr(ss, 'FusedSample', broken)
    with pytest.raises(HeliumError, match='out of memory'):
        ss.SurfaceSampler(Engine(), object(), object())
    assert ss.SurfaceSampler(Engine(), object(), object(), fused=False).fused is None
    # another surface object: its own frame() is used, through the three launches
    assert ss.SurfaceSampler(object(), object(), object()).fused is None
