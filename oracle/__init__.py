"""CPU oracle for the g_ab(r) / S_ab(Q) path (test infrastructure only; see orc.py)."""
