// Test infrastructure only: forwards to the Arith stand-in in vec.hxx.
#include <vec.hxx>
