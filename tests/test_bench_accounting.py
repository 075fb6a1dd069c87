"""CPU checks of the algorithmic counts bench.py reports beside its measured times (the
per-kernel bytes of the roofline table, the contraction's FMAs, the per-step bytes) at the
256 x 256 x 8 workload with 65,536 tracers."""
import pytest

import bench

NX = NY = 256
L = 8
CKEEP = 86          # columns c < 86 survive the 2/3 rule
NKEPT = CKEEP * 171  # kept rows: 85 below and 85 above the zero row, and the zero row
NTR = 65536


def test_contraction_fmas_per_point():
    # 20 units of L x ceil(L/2) coefficients and 38 edges of L + 1 FMAs, per output mode
    assert bench.contract_fmas_per_point(8) == 7856
    assert bench.contract_fmas_per_point(12) == 23208


def test_stage_bytes_at_the_workload():
    b = bench.stage_bytes(NX, NY, L, CKEEP, NKEPT, NTR)
    mb = {k: round(v / 1e6, 1) for k, v in b.items()}
    assert mb == {"synth_columns": 28.2, "rows_c2r": 56.1, "tracers": 24.1, "contract": 88.1,
                  "rows_r2c": 91.2, "columns_combine": 45.1, "update": 47.1}


def test_step_bytes_at_the_workload():
    step, tr = bench.bytes_alg(NX, NY, L, NTR)
    assert step == pytest.approx(319.8e6, rel=1e-3)
    assert tr == pytest.approx(74.4e6, rel=1e-3)
