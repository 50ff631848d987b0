"""avism_b200 -- B200 (sm_100a) library for the AVISM void-finding hot path."""
