// Environment flags of the drop-in interface (reference base/config.h:5-32).
#pragma once

#include <string>

class EnvironmentConfig
{
public:
    EnvironmentConfig(const EnvironmentConfig&) = delete;
    EnvironmentConfig(EnvironmentConfig&&)      = delete;
    static EnvironmentConfig& Get()
    {
        static EnvironmentConfig instance;
        return instance;
    }
    bool        showCurrentStep            = false;  // print solver progress
    bool        showGmresRes               = false;  // print the GMRES residual of each composite solve
    bool        track_pe_construct_time    = false;
    bool        track_pe_solve_detail_time = false;
    bool        track_pe_solve_total_time  = false;
    std::string pe_solve_total_name        = "pe_solve_total";

private:
    EnvironmentConfig() = default;
};
