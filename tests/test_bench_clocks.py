"""The bench's clock record: samples taken before the timed region (the
sampler starts before the warm-up) are left out of the reported median and
throttle reasons."""
import os
import time
from datetime import datetime

import bench


class _Done:
    def terminate(self):
        pass

    def wait(self):
        pass


def test_samples_before_mark_are_dropped(tmp_path):
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    t = time.time()
    rows = [(-5.0, 900, "Active"), (0.5, 1965, "Not Active"), (1.0, 1950, "Not Active")]
    with open(c.path, "w") as f:
        for dt, mhz, slow in rows:
            ts = datetime.fromtimestamp(t + dt).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
            f.write(f"{ts}, 0, {mhz}, 1965, 500.0, 0x0, {slow}, Not Active, Not Active, Not Active\n")
    c.proc, c.f, c.t_mark = _Done(), open(os.devnull, "w"), t
    out = c.stop()
    assert out["samples"] == 2
    assert out["sm_mhz"] == 1957.5
    assert out["reasons"] == []  # the hw_slowdown sample came before the mark
