from cola_halo_b200.schedule import Schedule, output_scale_factors, run_time_loop


def _events(sched, zout):
    ev = []
    run_time_loop(sched, output_scale_factors(zout), move=lambda: None, force=lambda: None,
                  kick=lambda a: None, drift=lambda a: None, snapshot=lambda a, i: None)
    return run_time_loop(sched, output_scale_factors(zout), move=lambda: None,
                         force=lambda: None, kick=lambda a: None, drift=lambda a: None,
                         snapshot=lambda a, i: ev.append(a))


def test_reference_schedule_counts():
    """main.c:71-72,145,162-206 with nsteps = 10, a_final = 1: 10 forces,
    9 kicks, 9 drifts, one snapshot at a = 1 after the 10th force."""
    ev = _events(Schedule.reference(10), [0.0])
    kinds = [e[0] for e in ev]
    assert kinds.count("force") == 10 and kinds.count("kick") == 9
    assert kinds.count("drift") == 9 and kinds[-1] == "snapshot"
    assert ev[0] == ("force", 0.1)


def test_linear_schedule_counts():
    ev = _events(Schedule.linear(0.02, 1.0, 10), [0.0])
    kinds = [e[0] for e in ev]
    assert kinds.count("force") == 11 and kinds.count("drift") == 10
    assert kinds[-1] == "snapshot"


def test_output_in_kick_window():
    """An output between apos0 and avel1 is written after the kick."""
    ev = _events(Schedule.reference(10), [1.0 / 0.52 - 1.0, 0.0])
    kinds = [e[0] for e in ev]
    i = kinds.index("snapshot")
    assert kinds[i - 1] == "kick"
