"""CPU oracle: test infrastructure, not product code.

A restatement of the reference's algorithms for the tracking path (C for the
pushers and the space-charge step, numpy for the map generator and the
learned-map network), each function citing the reference file:line it
follows, pinned against the golden vectors under tests/golden/.  Only the
tests, the smoke check and the benchmark's CPU-baseline legs may import it,
as the checker or as the timed CPU baseline; the tracking path never calls it
and fails loudly when its CUDA library is missing.
"""
