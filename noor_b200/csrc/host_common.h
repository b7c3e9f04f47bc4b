// Error reporting shared by the host parts of the library: every C-ABI call
// returns a NOOR_* status and leaves a message readable through
// noor_last_error() on the calling thread.
#pragma once
#include <string>

int set_error(int code, const std::string& msg);
void clear_error();
