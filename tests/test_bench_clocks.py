"""bench.Clocks keeps only the nvidia-smi samples written inside the timed region (between mark()
and stop()), and takes the next sample when the region was shorter than the sampling interval.
The sampler is faked: lines appended to its output file as nvidia-smi writes them."""
import threading
import time

import bench


class FakeSampler:
    def __init__(self):
        self.running = True

    def poll(self):
        return None if self.running else 0

    def terminate(self):
        self.running = False

    def wait(self):
        return 0


def line(sm, power_cap=False, thermal=False):
    act = lambda b: "Active" if b else "Not Active"
    return (f"0, {sm}, 1965, 700.00, 0x0, Not Active, Not Active, {act(thermal)}, {act(power_cap)}\n")


def make(tmp_path):
    c = object.__new__(bench.Clocks)
    c.path = str(tmp_path / "clocks.csv")
    c.proc = FakeSampler()
    c.first = 0
    return c


def test_only_the_samples_inside_the_region_count(tmp_path):
    c = make(tmp_path)
    with open(c.path, "w") as f:
        f.write(line(1100) + line(1100, thermal=True))  # before the region: idle, a thermal event
    c.mark()
    with open(c.path, "a") as f:
        f.write(line(1965) + line(1950, power_cap=True) + line(1965))
        f.write("0, 19")  # a line nvidia-smi has not finished
    got = c.stop()
    assert got == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_a_region_shorter_than_the_interval_takes_the_next_sample(tmp_path):
    c = make(tmp_path)
    with open(c.path, "w") as f:
        f.write(line(1100))
    c.mark()

    def later():
        time.sleep(0.1)
        with open(c.path, "a") as f:
            f.write(line(1965) + line(1965, thermal=True))

    t = threading.Thread(target=later)
    t.start()
    got = c.stop()
    t.join()
    assert got["samples"] == 1 and got["sm_mhz"] == 1965.0 and got["reasons"] == []


def test_no_sampler_gives_no_clocks(tmp_path):
    c = make(tmp_path)
    c.proc = None
    assert c.stop() is None
