"""Sharing the ensemble's boxes out over GPUs (bench.py --ensemble under torchrun): every box on
exactly one rank, and the largest per-rank load close to the ideal share."""
import pytest

import bench


@pytest.mark.parametrize("nranks", [1, 2, 3, 4, 8, 40])
def test_partition_covers_every_box_once(nranks):
    sizes = bench.ENSEMBLE_SIZES
    parts = bench.partition_boxes(sizes, nranks)
    assert len(parts) == nranks
    flat = sorted(b for p in parts for b in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[b] ** 3 for b in p) for p in parts]
    ideal = sum(s ** 3 for s in sizes) / nranks
    biggest = max(s ** 3 for s in sizes)
    assert max(loads) <= max(ideal * 1.35, biggest)
    assert bench.partition_boxes(sizes, nranks) == parts  # deterministic
