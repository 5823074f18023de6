// Entry points whose families are not built yet report so loudly.
#include "fast.h"
namespace ae {
}
