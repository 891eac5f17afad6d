// Stand-in for the termcolor header used by the ARTEA logger: every colour
// manipulator is a no-op, so log lines print uncoloured.
#pragma once
#include <ostream>

namespace termcolor {
inline std::ostream& reset(std::ostream& os) { return os; }
inline std::ostream& bold(std::ostream& os) { return os; }
inline std::ostream& grey(std::ostream& os) { return os; }
inline std::ostream& red(std::ostream& os) { return os; }
inline std::ostream& green(std::ostream& os) { return os; }
inline std::ostream& yellow(std::ostream& os) { return os; }
inline std::ostream& blue(std::ostream& os) { return os; }
inline std::ostream& magenta(std::ostream& os) { return os; }
inline std::ostream& cyan(std::ostream& os) { return os; }
inline std::ostream& white(std::ostream& os) { return os; }
inline std::ostream& on_red(std::ostream& os) { return os; }
inline std::ostream& underline(std::ostream& os) { return os; }
}  // namespace termcolor
