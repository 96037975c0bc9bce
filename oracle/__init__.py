"""Oracle package: CPU checkers for tests, smoke() and the CPU baseline. Test infrastructure only."""
