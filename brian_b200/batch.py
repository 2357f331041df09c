"""Batches of independent networks: many small Networks simulated side by
side in one kernel launch, one thread block per network.

The reference runs one Network per process (network.py:403-430 is the step
loop); a parameter study or an ensemble of seeds there is a loop over
networks.  ``NetworkBatch`` runs such a set at once on the GPU: each network
keeps its own connectivity, weights, parameters, initial state and duration
(uneven durations are allowed), and its results -- states, spike and state
monitor records, counters -- are those of ``Network.run`` on it alone, bit
for bit.  A network qualifies when it is one linear NeuronGroup of at most
4096 neurons and 1-4 variables without refractoriness, with at most two
shared-weight connections onto itself (zero-delay ``Connection`` or
``DelayConnection``), at most two undelayed SpikeMonitors and four
StateMonitors; the networks of a batch share the precision and the number
of state variables.  Others raise ``EngineError`` (code BG_ENOSYS) naming
the network and the reason.

    nets = [build(seed) for seed in range(256)]
    batch = NetworkBatch(nets)
    batch.autotune()                 # block shape and lanes per spike row
    batch.run([1 * second] * 256)    # or one duration for all
"""
from ._lib import BatchRuntime

__all__ = ["NetworkBatch"]


class NetworkBatch(object):
    def __init__(self, networks):
        self.networks = list(networks)
        if not self.networks:
            raise ValueError("empty batch")
        if len(set(id(n) for n in self.networks)) != len(self.networks):
            raise ValueError("a network appears twice in the batch")
        self._rt = None
        self._key = None
        self._shape = None

    def _runtime(self):
        for net in self.networks:
            net.prepare()
        key = tuple(id(net._binding) for net in self.networks)
        if self._rt is None or key != self._key:
            if self._rt is not None:
                self._rt.close()
            self._rt = BatchRuntime([net._binding.rt for net in self.networks])
            self._key = key
            if self._shape is not None:
                self._rt.set_shape(*self._shape)
        return self._rt

    def run(self, duration):
        """Run network i for duration[i] (or every network for one
        duration).  Networks that share a clock object must share the
        duration; each clock advances once."""
        durations = list(duration) if hasattr(duration, "__len__") else [duration] * len(self.networks)
        if len(durations) != len(self.networks):
            raise ValueError("one duration per network")
        rt = self._runtime()
        steps, cs0, clocks = [], [], {}
        for net, d in zip(self.networks, durations):
            k = net.clock.set_duration(d)
            prev = clocks.get(id(net.clock))
            if prev is not None and prev[1] != k:
                raise ValueError("networks sharing a clock need the same duration")
            clocks[id(net.clock)] = (net.clock, k)
            steps.append(k)
            cs0.append(net.clock.step)
        for net in self.networks:
            net.stopped = False
        rt.run(steps, cs0)
        for clock, k in clocks.values():
            clock._n += k

    def autotune(self, steps=200):
        """Time `steps` steps of every block shape and lanes-per-row setting
        without advancing any network and keep the fastest; returns its
        device time (ms)."""
        rt = self._runtime()
        ms = rt.autotune(steps)
        sh = rt.shape()
        self._shape = (sh["shape"], sh["lanes"])
        return ms

    def set_shape(self, shape, lanes=32):
        """Block shape index (128x4, 256x4, 512x4, 512x8, 1024x4, 768x6
        threads x neurons per thread) and lanes per spike row (4, 8, 16,
        32)."""
        self._runtime().set_shape(shape, lanes)
        self._shape = (int(shape), int(lanes))

    def shape(self):
        return self._runtime().shape()

    def stats(self):
        return self._runtime().stats()

    def close(self):
        if self._rt is not None:
            self._rt.close()
            self._rt = None
