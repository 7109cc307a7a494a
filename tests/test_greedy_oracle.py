"""The brute-force exact greedy that checks the device repair."""
import numpy as np

from oracle.dp_oracle import OracleBackend, exact_greedy


def test_exact_greedy_places_max_gain_smallest_index():
    ob = OracleBackend([3] * 5, 1)
    code = np.array([0, 100], dtype=np.int64)
    ob.recount(code)
    placed, deficit = exact_greedy(ob, code, 3)
    ob2 = OracleBackend([3] * 5, 1)
    cur = list(code)
    for w in placed:
        ob2.recount(np.array(cur))
        ob2.gain_map()
        g = ob2.map.astype(np.int64)
        g[np.array(cur)] = -1
        assert w == int(np.argmax(g))          # first maximum
        cur.append(int(w))
    ob2.recount(np.array(cur))
    assert deficit == ob2.uncovered()


def test_exact_greedy_stops_when_covered():
    ob = OracleBackend([3] * 4, 1)
    ob.recount(np.zeros(0, dtype=np.int64))
    placed, deficit = exact_greedy(ob, [], 10 ** 6)
    assert deficit == 0 and len(placed) == len(set(placed.tolist()))
