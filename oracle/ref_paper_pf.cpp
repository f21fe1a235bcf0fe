// ref_paper_pf.cpp -- the reference's example/paper/src/paper_pf.cpp model
// driven through vSMC's own Sampler (TEST INFRASTRUCTURE).
//
// Built by oracle/Makefile into oracle/_ref/ (git-ignored) from the example
// where it lies: the example's translation unit is included as it is, with
// its main() renamed, so its cv value type, cv_init, cv_move and
// cv_monitor_state are the reference's own.  The only code here is the
// driver of its main(), parameterised by particle count, steps, seed and the
// observation file.  Nothing in the product links it.
#define main vsmc_paper_pf_example_main
#include "paper_pf.cpp"
#undef main

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>

extern "C" {

// Seed::set(seed); Sampler<cv>(N, Stratified, 0.5) with cv_init, cv_move and
// the "pos" monitor as the example's main sets them up; initialize(data
// file) and iterate(T - 1).  The data file holds DataNum (100) rows of
// "x y".  Writes `os << sampler` into buf (at most cap bytes, NUL-
// terminated) and returns its full length.
uint64_t ref_paper_pf_summary (uint64_t N, uint64_t T, unsigned seed,
        const char *data_file, char *buf, uint64_t cap)
{
    vsmc::Seed::instance().set(seed);
    vsmc::Sampler<cv> sampler(N, vsmc::Stratified, 0.5);
    sampler.init(cv_init);
    sampler.move(cv_move(), false);
    vsmc::MonitorEvalAdapter<cv, vsmc::MonitorEvalSEQ> cv_est(
            cv_monitor_state);
    sampler.monitor("pos", 2, cv_est);
    std::vector<char> name(data_file, data_file + std::strlen(data_file) + 1);
    sampler.initialize(&name[0]);
    sampler.iterate(T - 1);
    std::stringstream ss;
    ss << sampler;
    const std::string text = ss.str();
    if (buf && cap > 0) {
        const uint64_t n = text.size() < cap - 1 ? text.size() : cap - 1;
        std::memcpy(buf, text.data(), n);
        buf[n] = '\0';
    }
    return text.size();
}

} // extern "C"
