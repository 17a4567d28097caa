"""trex_b200: B200-native (sm_100a) automaton simulation behind the TREX API."""
