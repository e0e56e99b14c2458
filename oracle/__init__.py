"""CPU oracle for the NTT / coset-LDE path -- test infrastructure only."""
