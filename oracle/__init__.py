"""Oracle test infrastructure (CPU).  Used only by tests/, the smoke check
and bench.py's CPU-baseline leg; never by the product path."""
