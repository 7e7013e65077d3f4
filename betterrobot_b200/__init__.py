"""B200-native (sm_100a) batched kinematics and LM-IK path with BetterRobot's call surface."""
