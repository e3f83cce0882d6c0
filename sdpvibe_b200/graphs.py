"""CUDA-graph replay of launch-bound call sequences (the batched Cholesky factorisation and the triangular
solves of ``mpf.Chol``).

A factorisation or a solve of given shapes is always the same sequence of a few hundred small launches
(residue GEMMs, CRTs, limb bookkeeping, base tiles) with no host decision that depends on the data, so
it is recorded once as a CUDA graph and replayed afterwards: the first call with a new key runs eagerly
(the library initialises its per-process state there) and then records the sequence on static copies of
its inputs; later calls copy their inputs into those buffers, replay, and return copies of the static
outputs (a result may be kept while the same graph runs again, e.g. the factors of X and of Y).  Replay
gives the same bits as the eager run: the same kernels run on the same data.  Replays of one graph from
different streams are ordered by an event (its static buffers are shared).

``SDPV_GRAPHS=0`` turns the replay off (every call eager).
"""
import os

import torch

from . import _trace

ENABLED = os.environ.get("SDPV_GRAPHS", "1") != "0"
_cache = {}


def _flatten(obj, out):
    """tensor leaves of obj in a fixed order (appended to out), and a hashable skeleton to rebuild it
    from new leaves"""
    if torch.is_tensor(obj):
        out.append(obj)
        return ("T",)
    if isinstance(obj, (list, tuple)):
        return (type(obj), tuple(_flatten(o, out) for o in obj))
    slots = getattr(type(obj), "__slots__", None)
    if slots:
        return ("S", type(obj), tuple((name, _flatten(getattr(obj, name), out)) for name in slots))
    return ("V", obj)                                   # int / None / str: kept as is (hashable)


def _rebuild(sk, it):
    kind = sk[0]
    if kind == "T":
        return next(it)
    if kind == "V":
        return sk[1]
    if kind == "S":
        obj = object.__new__(sk[1])
        for name, sub in sk[2]:
            setattr(obj, name, _rebuild(sub, it))
        return obj
    return kind(_rebuild(s, it) for s in sk[1])


class _Entry:
    __slots__ = ("graph", "inputs", "outputs", "skeleton", "launches", "done")


def run(key, fn, inputs):
    """fn(list of input tensors) -> result (tensors in lists / tuples / slotted objects).  The result of a
    replay is a fresh copy."""
    if not ENABLED or torch.cuda.is_current_stream_capturing():
        return fn(inputs)
    from .mpmat import moduli_group
    key = (key, moduli_group())                         # a graph holds the contexts it was recorded with
    e = _cache.get(key)
    if e is None:
        result = fn(inputs)                             # eager: also initialises lazy library state
        e = _Entry()
        e.inputs = [t.clone() for t in inputs]
        e.graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(e.graph), _trace.Trace() as rec:     # counts the recorded launches
            static = fn(e.inputs)
        e.launches = rec.launches
        e.done = None
        leaves = []
        e.skeleton = _flatten(static, leaves)
        e.outputs = leaves
        _cache[key] = e
        return result
    if e.done is not None:                              # a replay issued on another stream must be over
        torch.cuda.current_stream().wait_event(e.done)   # before its static buffers are written again
    for s, t in zip(e.inputs, inputs):
        s.copy_(t)
    end = _trace.replay(e.launches, _label(key))
    e.graph.replay()
    if end is not None:
        end.record()
    out = _rebuild(e.skeleton, iter([t.clone() for t in e.outputs]))
    if e.done is None:
        e.done = torch.cuda.Event()
    e.done.record()
    return out


def _label(key):
    """trace label of a graph: its key without the structure skeletons (plain values and integer shapes)"""
    keep = [k for k in key if not isinstance(k, tuple) or all(isinstance(x, int) for x in k)]
    return "graph " + " ".join(str(k) for k in keep)


def clear():
    """drop every recorded graph (and the memory its replays hold)"""
    _cache.clear()
