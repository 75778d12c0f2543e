"""CPU oracle of the BM25 Search path -- test infrastructure only (see oracle.py)."""
