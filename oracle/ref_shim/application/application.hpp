// Shim: the application logger is not used on the compiled path.
#pragma once
