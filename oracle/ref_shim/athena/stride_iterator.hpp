// Shim: Athena++'s stride iterator is not reached on the compiled path.
#pragma once
