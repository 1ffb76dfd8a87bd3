"""CPU restatement of viprs's resample path: test oracle and CPU baseline only."""
