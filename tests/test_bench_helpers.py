"""CPU checks of the bench's reference-baseline bookkeeping: the timings read
back from the reference's own log (timesys per plane, main.cpp:3455, and the
job's timesyshms total, main.cpp:3568)."""
import bench


def test_glg_times_reads_per_plane_and_total():
    text = ("Beginning grid calculations.\n"
            " 1    -10.000   1/3  Real= 0.12,  CPU= 0.10,  System= 0.00\n"
            " 2     -9.625   2/3  Real= 0.13,  CPU= 0.11,  System= 0.00\n"
            " 3     -9.250   3/3  Real= 0.25,  CPU= 0.20,  System= 0.01\n"
            "autogrid4: Successful Completion.\n"
            "Real= 1m 02.34s,  CPU= 3.00s,  System= 0.01s\n")
    t = bench.glg_times(text)
    assert t["planes"] == 3
    assert abs(t["plane_sum_s"] - 0.50) < 1e-9
    assert abs(t["real_total_s"] - 62.34) < 1e-9


def test_glg_times_hours_and_seconds_only():
    assert abs(bench.glg_times("Real= 1h 02m 03.50s,  CPU= 1.00s,")["real_total_s"] - 3723.5) < 1e-9
    assert abs(bench.glg_times("Real= 7.25s,  CPU= 7.00s,")["real_total_s"] - 7.25) < 1e-9
    assert bench.glg_times("no timings")["real_total_s"] is None


def test_cpu_model_is_text():
    assert isinstance(bench.cpu_model(), str) and bench.cpu_model()
