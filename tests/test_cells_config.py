"""The seeded uneven-cell workload generator (host only)."""
from megastation_b200 import datagen


def test_make_cells_shapes_and_seed():
    a = datagen.make_cells(n=32, seed=3)
    b = datagen.make_cells(n=32, seed=3)
    assert [vars(x) for x in a] == [vars(x) for x in b]
    for c in a:
        assert c.M in (32, 64, 128) and c.K in (4, 8, 16, 32) and c.K <= c.M
        assert datagen.CELL_SUBCARRIERS[c.S] == c.N
        assert c.Qm in (2, 4, 6) and 15.0 <= c.snr_db <= 25.0
        assert c.P + c.U == 14 and c.P * c.sg >= c.K
    assert len({(c.M, c.K, c.S, c.Qm) for c in a}) > 8
