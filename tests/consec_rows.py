"""Rows for the consecutive-frame merging tests (the generator lives in
qcstorm_b200.synth: blinking_rows, group_sizes)."""
from qcstorm_b200.synth import blinking_rows as consec_rows, group_sizes  # noqa: F401
