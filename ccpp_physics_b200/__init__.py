"""B200-native RRTMG longwave column path (drop-in for rrtmg_lw_run / rlwinit)."""
