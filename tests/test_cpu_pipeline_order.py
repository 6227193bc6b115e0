"""Ordering rules of the two-slot host pipeline (cortado_b200.pipeline), on the
CPU.  Streams and events are replaced by fakes that record what is enqueued;
the queues are then executed in many random interleavings that honour CUDA's
rules (a stream runs its operations in order; a wait blocks until the event's
record enqueued before the wait has executed).  In every interleaving:
item i runs after its copy in; its copy out starts after it ran; a slot's
next copy in starts only after the slot's previous run finished reading; and
a slot's next run starts only after its previous results were copied out."""
import random
import types

import pytest
import torch

from cortado_b200 import pipeline


class _Stream:
    def __init__(self, name):
        self.name = name
        self.ops = []

    def wait_event(self, ev):
        self.ops.append(("wait", ev, ev.version))

    def synchronize(self):
        pass


class _Event:
    def __init__(self):
        self.version = 0  # records enqueued so far

    def record(self, stream):
        self.version += 1
        stream.ops.append(("record", self, self.version))


def _fake_torch(cur):
    def stream_ctx(s):
        class _Ctx:
            def __enter__(self):
                cur.append(s)

            def __exit__(self, *a):
                cur.pop()
        return _Ctx()

    names = iter(["in", "out"])
    cuda = types.SimpleNamespace(Stream=lambda dev: _Stream(next(names)), Event=_Event, stream=stream_ctx)
    return types.SimpleNamespace(cuda=cuda, device=torch.device)


def _simulate(streams, rng):
    """Executes the queues in a random legal order; returns the sequence of
    (kind, item, 'start'|'end') with work split into start and end steps."""
    done_versions = {}
    pos = {s: 0 for s in streams}
    started = {}
    trace = []
    while True:
        ready = []
        for s in streams:
            if pos[s] >= len(s.ops):
                continue
            op = s.ops[pos[s]]
            if op[0] == "wait" and done_versions.get(id(op[1]), 0) < op[2]:
                continue
            ready.append(s)
        if not ready:
            break
        s = rng.choice(ready)
        op = s.ops[pos[s]]
        if op[0] == "record":
            done_versions[id(op[1])] = max(done_versions.get(id(op[1]), 0), op[2])
            pos[s] += 1
        elif op[0] == "wait":
            pos[s] += 1
        else:  # work: a start step, then an end step (other streams may run between)
            if not started.get((s, pos[s])):
                started[(s, pos[s])] = True
                trace.append((op[1], op[2], "start"))
            else:
                trace.append((op[1], op[2], "end"))
                pos[s] += 1
    assert all(pos[s] == len(s.ops) for s in streams), "deadlock: some queue never drained"
    return trace


@pytest.mark.parametrize("n_items", [1, 2, 3, 7])
def test_pipeline_ordering_rules(monkeypatch, n_items):
    cur = []
    monkeypatch.setattr(pipeline, "torch", _fake_torch(cur))
    slots = [types.SimpleNamespace(stream=_Stream("c0")), types.SimpleNamespace(stream=_Stream("c1"))]

    def work(kind):
        return lambda i, sl, s: cur[-1].ops.append(("work", kind, i))

    p = pipeline.Pipeline("cpu", slots, work("load"), work("run"), work("store"))
    p(n_items)
    p(n_items)  # a second batch of items on the same pipeline and events
    streams = [p.s_in, p.s_out] + [sl.stream for sl in slots]
    # each kind is enqueued on its own stream: loads on s_in, runs on the slot, stores on s_out
    assert {op[1] for op in p.s_in.ops if op[0] == "work"} <= {"load"}
    assert {op[1] for op in p.s_out.ops if op[0] == "work"} <= {"store"}
    for seed in range(200):
        trace = _simulate(streams, random.Random(seed))
        # the second batch reuses item numbers: tag each event with its batch
        seen, t = {}, {}
        for idx, (kind, i, ph) in enumerate(trace):
            b = seen.get((kind, i, ph), 0)
            seen[(kind, i, ph)] = b + 1
            t[(kind, b * 1000 + i, ph)] = idx
        items = [b * 1000 + i for b in range(2) for i in range(n_items)]
        for g in items:
            assert t[("load", g, "end")] < t[("run", g, "start")]
            assert t[("run", g, "end")] < t[("store", g, "start")]
        order = items  # global item order; slot = position % 2 within each batch
        for a_idx, a in enumerate(order):
            for b in order[a_idx + 1:]:
                if (a % 1000) % 2 != (b % 1000) % 2:
                    continue
                # b reuses a's slot: its copy in waits for a's run, its run for a's copy out
                assert t[("run", a, "end")] < t[("load", b, "start")]
                assert t[("store", a, "end")] < t[("run", b, "start")]
