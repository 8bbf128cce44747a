"""Serving loop (continuous batching) on the GPU: every request's result is
the same alone and in the mix, requests admitted while others are running
join the shared scan, and admission, cancellation and bounded waits behave
on the host side."""
import threading
import time

import numpy as np
import pytest

import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = 2_000_003  # not a multiple of the segment or of 32


@pytest.fixture(scope="module")
def table():
    cols = [D.uniform(N, 1), D.zipf(N, 2, 1.3), D.uniform(N, 3, 256), D.normal(N, 4)]
    return cols


def alone(ctx, q):
    """The single-query fused scan of q (the reference result for the mix)."""
    words = R.bitmap_words(ctx.nrows)
    bm = torch.empty(words, dtype=torch.int32, device="cuda")
    cnt = torch.empty(1, dtype=torch.int64, device="cuda")
    ctx.scan_async(q, bm.data_ptr(), cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return bm.cpu().numpy().view(np.uint32).copy(), int(cnt.item())


def test_results_alone_and_in_the_mix(ctx, table):
    ctx.load_columns(table)
    qs = D.batch_queries(table, 300, seed=1)
    qs += [[], [(1, 5, 4)], [(c, 0, 0xFFFFFFF0) for c in range(4)]]   # outside-the-kernel requests
    want = [alone(ctx, q) for q in qs]
    with R.Server(ctx, max_active=64, segment_rows=1 << 18) as srv:
        tickets = [None] * len(qs)

        def producer(lo, hi, delay):
            for i in range(lo, hi):
                tickets[i] = srv.submit(qs[i])
                if delay:
                    time.sleep(delay)

        # three producers, one of them trickling so arrivals land while others run
        th = [threading.Thread(target=producer, args=(0, 100, 0)),
              threading.Thread(target=producer, args=(100, 200, 0.0005)),
              threading.Thread(target=producer, args=(200, len(qs), 0))]
        for t in th:
            t.start()
        # consume results in completion order while the producers run: a done
        # result holds its slot until fetched, so waiting in submission order
        # could leave every slot held by results nobody reads yet
        pending = set(range(len(qs)))
        deadline = time.time() + 120
        while pending and time.time() < deadline:
            progress = False
            for i in list(pending):
                if tickets[i] is None:
                    continue
                done, _ = srv.poll(tickets[i])
                if done:
                    bm, cnt = srv.fetch(tickets[i])
                    assert cnt == want[i][1], (i, qs[i])
                    assert np.array_equal(bm, want[i][0]), (i, qs[i])
                    pending.discard(i)
                    progress = True
            if not progress:
                time.sleep(0.001)
        for t in th:
            t.join()
        assert not pending
        st = srv.stats()
        assert st["completed"] == len(qs)
        assert st["steps"] > 0
        assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]


def test_served_result_matches_oracle(ctx, table):
    ctx.load_columns(table)
    qs = D.batch_queries(table, 12, seed=7)
    with R.Server(ctx, max_active=8, segment_rows=1 << 19) as srv:
        tks = [srv.submit(q) for q in qs]
        for q, tk in zip(qs, tks):
            srv.wait(tk)
            bm, cnt = srv.fetch(tk)
            ref, rcnt = O.range_scan([table[c] for c, _, _ in q], [t[1] for t in q], [t[2] for t in q])
            assert cnt == rcnt and np.array_equal(bm, ref)


def test_queue_full_cancel_and_timeout(ctx, table):
    ctx.load_columns(table)
    q = [(0, 1 << 30, 3 << 30), (1, 0, 100)]
    with R.Server(ctx, max_active=2, max_queue=4, segment_rows=1 << 16) as srv:
        accepted, full = [], 0
        for _ in range(40):
            try:
                accepted.append(srv.submit(q))
            except R.RtsError as e:
                assert e.code == -8
                full += 1
        assert full > 0
        # a bounded wait that runs out returns an error, and the server goes on
        with pytest.raises(R.RtsError) as e:
            srv.wait(accepted[-1], 0)
        assert e.value.code == -7
        srv.cancel(accepted[-1])
        counts = []
        for tk in accepted[:-1]:
            srv.wait(tk, 60000)
            counts.append(srv.fetch(tk, want_bitmap=False)[1])
        st = srv.stats()
        assert st["cancelled"] == 1 and st["rejected"] == full
    ocnt = O.range_scan([table[0], table[1]], [1 << 30, 0], [3 << 30, 100])[1]
    assert counts and all(c == ocnt for c in counts)
    # after the server stops the context is usable again
    assert alone(ctx, q)[1] == ocnt


def test_replay_open_loop(ctx, table):
    ctx.load_columns(table)
    qs = D.batch_queries(table, 400, seed=9)
    rng = np.random.default_rng(0)
    arrivals = np.cumsum(rng.exponential(1 / 20000.0, size=len(qs)))  # 20k q/s Poisson
    with R.Server(ctx, max_active=256, segment_rows=1 << 18) as srv:
        lat = srv.replay(qs, arrivals)
        assert (lat > 0).all()
        st = srv.stats()
        assert st["completed"] == len(qs)


def test_replay_stopped_by_a_refused_request_releases_its_slots(ctx, table):
    """A replay that stops partway (here the server refuses a request whose
    column does not exist) cancels its requests still in flight: no result
    slot stays held, and the server answers later requests in full."""
    ctx.load_columns(table)
    good = D.batch_queries(table, 40, seed=11)
    qs = good[:25] + [[(99, 0, 10)]] + good[25:]
    arrivals = np.linspace(0, 0.01, len(qs))
    with R.Server(ctx, max_active=8, segment_rows=1 << 18) as srv:
        with pytest.raises(R.RtsError) as e:
            srv.replay(qs, arrivals)
        assert e.value.code == -1  # RTS_ERR_ARG, the refused submit
        assert srv.stats()["active"] == 0
        # every slot is free again: max_active requests run at once
        tks = [srv.submit(q) for q in good[:8]]
        for q, tk in zip(good[:8], tks):
            srv.wait(tk, 60000)
            assert srv.fetch(tk, want_bitmap=False)[1] == alone(ctx, q)[1]
        lat = srv.replay(good, np.linspace(0, 0.01, len(good)))
        assert (lat > 0).all()


def test_cancels_while_running_and_slots_reused(ctx, table):
    """Requests cancelled while the scan runs them leave the running plan
    without a re-plan; their slots are reused by later requests, whose
    results (and every request not cancelled) equal the direct scan."""
    ctx.load_columns(table)
    qs = D.batch_queries(table, 240, seed=13)
    want = [alone(ctx, q) for q in qs]
    rng = np.random.default_rng(3)
    with R.Server(ctx, max_active=24, segment_rows=1 << 17) as srv:
        live = {}
        cancelled = 0
        for i, q in enumerate(qs):
            live[srv.submit(q)] = i
            if i % 3 == 2:  # cancel one of the requests submitted so far, running or queued
                tk = list(live)[int(rng.integers(0, len(live)))]
                try:
                    srv.cancel(tk)
                    live.pop(tk)
                    cancelled += 1
                except R.RtsError:
                    pass  # already being fetched below, or done and released
            # fetch whatever is done, so that slots free up for new requests
            for tk in list(live):
                done, _ = srv.poll(tk)
                if done:
                    bm, cnt = srv.fetch(tk)
                    j = live.pop(tk)
                    assert cnt == want[j][1] and np.array_equal(bm, want[j][0]), j
        for tk, j in list(live.items()):
            srv.wait(tk, 120000)
            bm, cnt = srv.fetch(tk)
            assert cnt == want[j][1] and np.array_equal(bm, want[j][0]), j
        st = srv.stats()
        assert st["cancelled"] == cancelled > 0
        assert st["active"] == 0


def test_many_active_requests_share_positions(ctx, table):
    """600 requests over the four columns running at once make table passes
    that share one position search per segment row (the server's segment
    scratch); every result equals the direct scan."""
    ctx.load_columns(table)
    qs = D.batch_queries(table, 600, seed=17, min_cols=2, max_cols=4)
    want = [alone(ctx, q) for q in qs]
    with R.Server(ctx, max_active=1024, segment_rows=1 << 18) as srv:
        tks = [srv.submit(q) for q in qs]
        for i, tk in enumerate(tks):
            srv.wait(tk, 120000)
            bm, cnt = srv.fetch(tk)
            assert cnt == want[i][1] and np.array_equal(bm, want[i][0]), i
        assert srv.stats()["plans"] >= 1
