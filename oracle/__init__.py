"""CPU oracle for the ddCOSMO path (test infrastructure only; see ddc_ref.c)."""
