"""kw_run streams large recorded time series to the host while the loop runs.

The chunked copy (a copy stream into a pinned ring, drained into the caller's
buffers while the GPU computes the next chunk) must return exactly what the
split form returns: kw_run_device followed by kw_copy_outputs on the same plan.
"""
import numpy as np
import pytest


def _problem(kw, N=512, Nt=600, start=101):
    kg = kw.kWaveGrid(N, 1e-4, N, 1e-4)
    kg.setTime(Nt, 0.3 * 1e-4 / 1600.0)
    ax = np.arange(N)
    c = 1500.0 + 100.0 * np.exp(-((ax[:, None] - N / 3) ** 2 + (ax[None, :] - N / 2) ** 2) / (2 * 30.0 ** 2))
    medium = {"sound_speed": c, "density": 1000.0 + 0.6 * (c - 1500.0), "alpha_coeff": 0.5, "alpha_power": 1.5}
    p0 = kw.makeDisc(N, N, N // 2, N // 2, 6)
    mask = np.zeros((N, N))
    mask[:, N // 2 - 32:N // 2 + 32] = 1          # 32768 points
    # p, ux, uy: 3 x 32768 x 500 x 4 B = 197 MB, streamed in chunks of 42 steps
    sensor = {"mask": mask, "record": ["p", "u", "p_max", "p_rms"], "record_start_index": start}
    return kg, medium, {"p0": p0}, sensor


@pytest.mark.gpu
def test_streamed_series_equal_split_copy():
    import kwave_b200 as kw
    kg, med, src, sen = _problem(kw)
    with kw.Simulation(2, kg, med, src, sen, PMLSize=16) as sim:
        streamed = sim.run()
        sim.run_device()
        split = sim.copy_outputs()
        again = sim.run()
    assert set(streamed) == set(split)
    for k in split:
        assert streamed[k].shape == split[k].shape, k
        assert np.array_equal(streamed[k], split[k]), k
        assert np.array_equal(again[k], split[k]), k
    assert streamed["p"].shape == (512 * 64, 500)
    assert np.abs(streamed["p"]).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [True, 7])
def test_stream_to_disk_equals_plain_run(tmp_path, monkeypatch, steps):
    """StreamToDisk: the p series goes through a device buffer of `steps`
    columns and the reference's temp_sensor_data.bin in the working
    directory, and comes back identical to the plain run; the file is gone
    afterwards (kspaceFirstOrder3D.m:1101-1146, 1235-1295).  7 does not divide
    the 160 recorded steps, so the last chunk is partial."""
    import kwave_b200 as kw
    monkeypatch.chdir(tmp_path)
    N = 48
    kg = kw.kWaveGrid(N, 1e-4, N, 1e-4, N, 1e-4)
    kg.setTime(180, 0.3 * 1e-4 / 1600.0)
    ax = np.arange(N)
    c = 1500.0 + 100.0 * np.exp(-((ax[:, None, None] - 20) ** 2 + (ax[None, :, None] - 24) ** 2
                                  + (ax[None, None, :] - 28) ** 2) / (2 * 6.0 ** 2))
    med = {"sound_speed": c, "density": 1000.0, "alpha_coeff": 0.5, "alpha_power": 1.5}
    mask = np.zeros((N, N, N))
    mask[30, :, :] = 1
    src = {"p0": kw.makeBall(N, N, N, 24, 24, 24, 4)}
    sen = {"mask": mask, "record_start_index": 21}
    plain = kw.kspaceFirstOrder3D(kg, med, src, sen, PMLSize=6)
    streamed = kw.kspaceFirstOrder3D(kg, med, src, sen, PMLSize=6, StreamToDisk=steps)
    assert streamed.shape == plain.shape == (N * N, 160)
    assert np.array_equal(streamed, plain)
    assert not (tmp_path / "temp_sensor_data.bin").exists()
