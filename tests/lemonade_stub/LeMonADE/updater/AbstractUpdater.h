// Test stand-in for LeMonADE's updater base class (LeMonADE is not installed here): only what
// include/bfm_lemonade.hpp and the reference's adapter (src/pscbfm/GPUScBFM_AB_Type.h) use, so that
// both adapters' code is compiled by the test suite.
#pragma once

class AbstractUpdater
{
public:
    virtual ~AbstractUpdater() = default;
    virtual void initialize() = 0;
    virtual bool execute() = 0;
    virtual void cleanup() = 0;
};
