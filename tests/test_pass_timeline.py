"""The pass-timeline summary (medyan_b200.pass_timeline) on synthetic block
records: per-kernel first start, last end, last start and block durations
relative to the pass's first block. No GPU: the records are made here."""
import numpy as np

from medyan_b200.pass_timeline import REC, summarize


def test_summary_of_synthetic_records():
    r = np.zeros(5, dtype=REC)
    # kind, block, start and end in ns on the global timer
    rows = [(3, 0, 1000, 2000), (3, 1, 1100, 2500), (0, 0, 3000, 9000), (0, 1, 4000, 8000), (200, 0, 9000, 9500)]
    for i, (kind, blk, t0, t1) in enumerate(rows):
        r[i]["kind"], r[i]["block"], r[i]["t0"], r[i]["t1"] = kind, blk, t0, t1
    lines = summarize(r)
    assert lines[0] == "5 records, span 8.5 us"
    zero = next(line for line in lines if line.strip().startswith("zero"))
    assert "blocks     2" in zero and "start    0.0" in zero and "end    1.5" in zero and "last start    0.1" in zero
    main = next(line for line in lines if line.strip().startswith("main.forces"))
    # block durations 6 and 4 us: median 5
    assert "start    2.0" in main and "end    8.0" in main and "median  5.00" in main and "max   6.00" in main
    assert any(line.strip().startswith("finish.main") for line in lines)
