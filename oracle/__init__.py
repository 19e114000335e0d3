"""ORACLE — test infrastructure only: the float64 CPU restatement of the reference's CPU hydro
scheme. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import it."""
