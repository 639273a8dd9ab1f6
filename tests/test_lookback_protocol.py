"""The decoupled look-back protocol of the two-way partition behind
Partition512 (s512_partition2.cuh), simulated with host threads (no GPU):
tiles take chain positions in the order they start, publish their aggregate,
walk back to the nearest inclusive count with a bounded wait, and publish
their inclusive count.  The prefixes must equal a serial scan, and a tile that
never publishes must make its successors time out, not hang."""
import random
import threading

AGG, INC = 1 << 62, 1 << 63
VAL = (1 << 62) - 1


def run(counts, window=8, spin_limit=200000, dead=None):
    n = len(counts)
    status = [0] * n
    lock = threading.Lock()
    chain = [0]
    prefixes = [None] * n
    timeouts = [0]

    def worker():
        while True:
            with lock:
                pos = chain[0]
                chain[0] += 1
            if pos >= n:
                return
            if pos == dead:
                continue  # this tile never publishes anything
            h = counts[pos]
            status[pos] = (INC if pos == 0 else AGG) | h
            prefix = 0
            if pos > 0:
                p = pos - 1
                done = ok = False
                while not done and ok is False:
                    ok = None
                    for w in range(window):
                        q = p - w
                        if q < 0:
                            break
                        spins = 0
                        while not status[q] & (INC | AGG):
                            spins += 1
                            if spins > spin_limit:
                                break
                        v = status[q]
                        if not v & (INC | AGG):
                            timeouts[0] += 1
                            done = True
                            prefix = None
                            break
                        prefix += v & VAL
                        if v & INC:
                            done = True
                            break
                    p -= window
                    if ok is None and not done:
                        ok = False
                if prefix is not None:
                    status[pos] = INC | (prefix + h)
                else:
                    status[pos] = INC | h  # successors learn a wrong prefix; the error is reported
            prefixes[pos] = prefix

    threads = [threading.Thread(target=worker) for _ in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=60)
        assert not t.is_alive(), "a simulated tile hung"
    return prefixes, timeouts[0]


def test_prefixes_equal_serial_scan():
    rng = random.Random(1)
    counts = [rng.randrange(0, 300) for _ in range(2000)]
    prefixes, timeouts = run(counts)
    assert timeouts == 0
    acc = 0
    for i, c in enumerate(counts):
        assert prefixes[i] == acc
        acc += c


def test_missing_tile_times_out_instead_of_hanging():
    counts = [5] * 64
    prefixes, timeouts = run(counts, spin_limit=2000, dead=10)
    assert timeouts >= 1
    assert prefixes[10] is None
