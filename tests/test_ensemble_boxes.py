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
