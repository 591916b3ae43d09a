"""The launch-configuration autotuner (host logic; the timer is faked so the
test needs no GPU): fastest candidate wins, choices are cached per shape and
persisted, and disabling tuning returns the default."""
import json

from emustack_b200.autotune import Autotuner, size_bucket


def fake_timer(times, calls):
    def t(run, c, stream):
        calls.append(c)
        run(c)
        return times[c]
    return t


def test_fastest_choice_is_cached_and_persisted(tmp_path, monkeypatch):
    monkeypatch.delenv('EMUSTACK_AUTOTUNE', raising=False)
    path = str(tmp_path / 'tune.json')
    calls, ran = [], []
    at = Autotuner(path=path, time_fn=fake_timer({0: 3.0, 1: 1.5, 2: 2.0}, calls))
    c = at.choose('film_stack', {'L': 12, 'npw': 81}, [0, 1, 2], ran.append, 0)
    assert c == 1 and sorted(calls) == [0, 1, 2]
    # second call: no timing
    assert at.choose('film_stack', {'npw': 81, 'L': 12}, [0, 1, 2], ran.append, 0) == 1
    assert len(calls) == 3
    # another shape is tuned separately
    assert at.choose('film_stack', {'L': 4, 'npw': 81}, [0, 1, 2], ran.append, 0) == 1
    assert len(calls) == 6
    saved = json.load(open(path))
    assert len(saved) == 2 and all(v['choice'] == 1 for v in saved.values())
    # a new tuner reads the file and does not time again
    calls2 = []
    at2 = Autotuner(path=path, time_fn=fake_timer({0: 0.1, 1: 9.0, 2: 9.0}, calls2))
    assert at2.choose('film_stack', {'L': 12, 'npw': 81}, [0, 1, 2], ran.append, 0) == 1
    assert calls2 == []


def test_tuple_choices_and_disable(monkeypatch):
    calls = []
    at = Autotuner(path='', time_fn=fake_timer({(4096, 2): 2.0, (8192, 4): 1.0}, calls))
    assert at.choose('overlap_tc', {'npw': 309}, [(4096, 2), (8192, 4)], lambda c: None, (4096, 2)) == (8192, 4)
    monkeypatch.setenv('EMUSTACK_AUTOTUNE', '0')
    off = Autotuner(path='', time_fn=fake_timer({}, []))
    assert off.choose('x', {}, [1, 2], lambda c: None, 7) == 7


def test_size_bucket():
    assert [size_bucket(n) for n in (0, 1, 2, 3, 4, 5, 32768, 32769)] == [1, 1, 2, 4, 4, 8, 32768, 65536]


def test_failing_candidate_is_skipped():
    def t(run, c, stream):
        if c == 2:
            raise RuntimeError('launch failed')
        return {0: 2.0, 1: 3.0}[c]
    at = Autotuner(path='', time_fn=t)
    assert at.choose('film_stack', {'L': 3}, [0, 1, 2], lambda c: None, 0) == 0


def test_near_ties_keep_the_first_candidate():
    """Candidates within 2 % of the fastest count as a tie, and the first of
    them in the caller's order wins, so noise does not flip the choice."""
    from emustack_b200.autotune import Autotuner
    ms = {0: 2.50, 1: 3.90, 4: 2.44, 5: 2.40}
    t = Autotuner(path='', time_fn=lambda run, c, s: ms[c])
    assert t.choose('k', {'n': 1}, [0, 1, 4, 5], lambda c: None, 0) == 4   # 2.44 within 2 % of 2.40, 2.50 not
    ms2 = {0: 2.44, 1: 3.90, 4: 2.46, 5: 2.40}
    t2 = Autotuner(path='', time_fn=lambda run, c, s: ms2[c])
    assert t2.choose('k', {'n': 1}, [0, 1, 4, 5], lambda c: None, 0) == 0
