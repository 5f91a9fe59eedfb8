// ORACLE shim (test infrastructure): serialization is not exercised.
#pragma once
namespace boost { namespace serialization { class access; } }
