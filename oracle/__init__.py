"""CPU oracle of the sortArray path. Test infrastructure only: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg."""
