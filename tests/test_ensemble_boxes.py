"""The ensemble workload's boxes (host-side generator, no GPU needed)."""
from filsim_b200.ensemble import filament_cap, make_boxes


def test_filament_caps():
    assert [filament_cap(n) for n in (48, 64, 96, 128)] == [12, 30, 102, 243]


def test_ensemble_workload_draw():
    boxes = make_boxes(3, nboxes=8)
    for npts, p, s, kb in boxes:
        assert npts in (48, 64, 96, 128)
        assert 1 <= s.nfil <= filament_cap(npts)
        assert 0.1 <= kb <= 10.0
        assert s.np == 16 * s.nfil


def test_partition_over_ranks():
    """partition_boxes: every box on exactly one rank, the largest-first greedy split
    leaves no rank more than one box's cost above the lightest, and one rank takes all."""
    from filsim_b200.ensemble import box_cost, partition_boxes
    boxes = make_boxes(11, nboxes=24)
    cost = [box_cost(npts, s.np) for npts, _, s, _ in boxes]
    assert partition_boxes(boxes, 1) == [list(range(24))]
    for world in (2, 3, 4, 8):
        parts = partition_boxes(boxes, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(24))
        loads = [sum(cost[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cost)
        assert partition_boxes(boxes, world) == parts  # deterministic: every rank computes the same split
