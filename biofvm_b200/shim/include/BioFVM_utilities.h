// Stopwatch helpers with BioFVM's names (BioFVM_utilities.h).  The reference
// times with clock() (CPU time summed over threads); these report wall time.
#ifndef __BioFVM_utilities_h__
#define __BioFVM_utilities_h__

#include <cmath>
#include <ctime>
#include <iostream>
#include <string>

namespace BioFVM {
void TIC(void);
void TOC(void);
void RUNTIME_TIC(void);
void RUNTIME_TOC(void);
double stopwatch_value(void);
double runtime_stopwatch_value(void);
double total_stopwatch_time(void);
void display_stopwatch_value(std::ostream& os, double dIn);
std::string format_stopwatch_value(double dIn);
}  // namespace BioFVM

#endif
