/* Links against tapp::reference through the CMake package and makes the
 * calls a consumer's smoke test makes: handle, executor, error text. */
#include <stdio.h>
#include <stdlib.h>
#include <tapp.h>

int main(void)
{
    TAPP_handle h;
    TAPP_executor e;
    if (!TAPP_check_success(TAPP_create_handle(&h)) || !TAPP_check_success(TAPP_create_executor(&e))) return 1;
    char msg[128];
    TAPP_explain_error(1, sizeof msg, msg);
    if (!TAPP_check_success(TAPP_destroy_executor(e)) || !TAPP_check_success(TAPP_destroy_handle(h))) return 1;
    printf("consume ok: %s\n", msg);
    return EXIT_SUCCESS;
}
