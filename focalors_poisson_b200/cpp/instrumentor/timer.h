// Scope timers of the drop-in interface: the reference's SCOPE_TIMER / FUNCTION_TIMER macros
// (instrumentor/timer.h:96-103) as host wall-clock timers that print when asked to.
#pragma once

#include <chrono>
#include <iostream>
#include <string>

enum TimeRecordType : unsigned char
{
    None,
    List,
    Accumulate
};

class Timer
{
public:
    Timer(const std::string& name, TimeRecordType, bool output)
        : name_(name), output_(output), t0_(std::chrono::steady_clock::now())
    {}
    ~Timer() { Stop(); }
    void Stop()
    {
        if (stopped_) return;
        stopped_ = true;
        if (output_)
            std::cout << name_ << " "
                      << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count() << "s"
                      << std::endl;
    }

private:
    std::string                           name_;
    bool                                  output_;
    bool                                  stopped_ = false;
    std::chrono::steady_clock::time_point t0_;
};

#define SCOPE_TIMER_LINE(name, line, type, output)      Timer timer##line(name, type, output)
#define SCOPE_TIMER_PASTELINE(name, line, type, output) SCOPE_TIMER_LINE(name, line, type, output)
#define SCOPE_TIMER(name, type, output)                 SCOPE_TIMER_PASTELINE(name, __LINE__, type, output)
#define FUNCTION_TIMER(type, output)                    SCOPE_TIMER(__PRETTY_FUNCTION__, type, output)
