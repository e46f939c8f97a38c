"""FP64 CPU oracle for the resist-shrinkage operator (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs as the checker; the product package never imports it."""
