"""CPU oracles of the reference's algorithms: test infrastructure only (see ``oracle/bloch.py``)."""
