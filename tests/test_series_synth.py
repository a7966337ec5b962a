"""The advected tracer series (the uneven time-series workload) on the CPU:
the velocity field is divergence-free, the advection is deterministic and
smooth, and the frames have the workload's shapes."""
import numpy as np


def test_velocity_field_is_divergence_free(synthmod):
    rng = np.random.default_rng(0)
    pos = rng.random((2000, 3))
    for seed in (0, 1, 7):
        f = synthmod.velocity_modes(seed)
        u = synthmod.velocity(pos, f)
        assert np.abs(synthmod.divergence(pos, f)).max() < 1e-12 * max(1.0, np.abs(u).max())
        # and by central differences, independently of the analytic form
        h = 1e-5
        div = np.zeros(len(pos))
        for j in range(3):
            e = np.zeros(3)
            e[j] = h
            div += (synthmod.velocity(pos + e, f)[:, j] - synthmod.velocity(pos - e, f)[:, j]) / (2 * h)
        assert np.abs(div).max() < 1e-6 * np.abs(u).max() * 2 * np.pi * 6


def test_tracers_are_advected_deterministically(synthmod):
    a = synthmod.tracer_positions(0, 5)
    b = synthmod.tracer_positions(0, 5)
    assert np.array_equal(a, b)
    assert a.shape == (synthmod.SERIES_TRACERS, 3) and a.min() >= 0 and a.max() < 1
    # consecutive frames move every tracer a little (periodic distance)
    d = synthmod.tracer_positions(0, 6) - a
    d = np.abs(d - np.round(d))
    step = np.linalg.norm(d, axis=1)
    assert 0 < np.median(step) < 0.05 and step.max() < 0.1
    assert not np.array_equal(synthmod.tracer_positions(1, 5), a)


def test_series_frames_have_the_workload_shapes(synthmod):
    frames = synthmod.series_frames(64)
    assert len(frames) == 64
    for i, c in enumerate(frames):
        assert c.W in (512, 640, 768, 1024) and c.H == c.W
        assert 100 <= c.num_planes <= 400 and 200 <= c.n_disks <= 3000
        assert (c.plane_stepsize, c.resolution, c.wavelength) == (2.0, 1.1, 0.632)
        assert c.series_frame == i
    assert len({c.W for c in frames}) == 4 and len({c.num_planes for c in frames}) > 30  # uneven sizes
    # frame masks are built from the advected population
    c = synthmod.series_frames(2)[1]
    c.width = c.height = 64
    c.num_planes = 10
    c.n_disks = 40
    masks = synthmod.object_masks(c)
    assert sum(int(m.sum() > 0) for m in masks.values()) > 0
