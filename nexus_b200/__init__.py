"""nexus_b200: a B200-native (sm_100a) MLS-MPM step with nexus_mpm's API."""
