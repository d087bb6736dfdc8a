"""The N > 1 path on CPU: world-size-2 gloo process groups (127.0.0.1).

Each rank renders its row band of one frame with the oracle; the bands
gathered to rank 0 equal a single full-frame render bit for bit (strong
scaling by rows), the max-over-ranks timing reduction returns the slowest
rank, and weak-scaling seeds differ per rank."""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from oracle.oracle import OracleFilm
        from psycles_b200 import _abi, dist as pdist, scenes
        scene = scenes.small_test_scene(seed=2)
        w, h = 40, 30
        first, rows = pdist.row_band(rank, world, h)
        st = scenes.render_settings(w, h, max_bounces=3, window_y=first, window_height=rows)
        film = OracleFilm(st)
        film.render(scene.to_desc(), 0, 3, 3, threads=1)
        band = film.resolve(_abi.PASS_COMBINED)
        frame = pdist.gather_bands(band, h)
        slowest = pdist.max_over_ranks(float(rank + 1) * 10.0)
        if rank == 0:
            np.save(os.path.join(out_dir, "frame.npy"), frame)
            np.save(os.path.join(out_dir, "slowest.npy"), np.array([slowest]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_row_bands_partition_the_frame():
    from psycles_b200 import dist as pdist
    for world in (1, 2, 3, 8):
        for h in (1, 7, 30, 1080):
            bands = [pdist.row_band(r, world, h) for r in range(world)]
            covered = [y for f, n in bands for y in range(f, f + n)]
            assert covered == list(range(h))
            assert max(n for _, n in bands) - min(n for _, n in bands) <= 1
    assert {pdist.frame_seed(r) for r in range(8)} == set(range(8))


def test_two_rank_row_split_equals_full_frame(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    from oracle.oracle import OracleFilm
    from psycles_b200 import _abi, scenes
    scene = scenes.small_test_scene(seed=2)
    st = scenes.render_settings(40, 30, max_bounces=3)
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 3, 3, threads=1)
    full = film.resolve(_abi.PASS_COMBINED)
    frame = np.load(tmp_path / "frame.npy")
    assert np.array_equal(frame.view(np.uint32), full.view(np.uint32))
    assert float(np.load(tmp_path / "slowest.npy")[0]) == 20.0
