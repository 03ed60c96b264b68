// Test stand-in for LeMonADE's updater base class (LeMonADE is not installed here): only what
// include/bfm_lemonade.hpp uses, so that the adapter's code is compiled by the test suite.
#pragma once

class AbstractUpdater
{
public:
    virtual ~AbstractUpdater() = default;
    virtual void initialize() = 0;
    virtual bool execute() = 0;
    virtual void cleanup() = 0;
};
